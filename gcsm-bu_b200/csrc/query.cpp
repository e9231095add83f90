#include "query.h"

#include <algorithm>
#include <map>

namespace csm {

std::string build_query(uint32_t nv, const uint32_t *vlabel, uint32_t ne, const uint32_t *src,
                        const uint32_t *dst, const uint32_t *elabel, Query &q) {
    // Size limits of utils/config.h:9-10 and the vcount_ >= 2 rule of graph.cpp:264-268.
    if (nv < 2) return "the number of query vertices should not be less than 2";
    if (nv > 16 || ne > 42) return "the query graph should have at most 16 vertices and 42 edges";
    if (ne == 0) return "the query graph has no edge";
    q = Query();
    q.nv = nv;
    q.ne = ne;
    q.vlabel.assign(vlabel, vlabel + nv);
    q.nbrs.assign(nv, {});
    q.qe_index.assign(nv * nv, -1);
    for (uint32_t e = 0; e < ne; e++) {
        uint32_t a = src[e], b = dst[e];
        if (a >= nv || b >= nv) return "query edge endpoint out of range";
        if (a == b) return "query self-loops are not supported";
        for (auto &p : q.nbrs[a])
            if (p.first == b) return "parallel query edges are not supported";
        // Sorted insertion, as graph.cpp:251-258.
        auto pa = std::make_pair(b, elabel[e]);
        q.nbrs[a].insert(std::lower_bound(q.nbrs[a].begin(), q.nbrs[a].end(), pa), pa);
        auto pb = std::make_pair(a, elabel[e]);
        q.nbrs[b].insert(std::lower_bound(q.nbrs[b].begin(), q.nbrs[b].end(), pb), pb);
    }
    // qe_list_ order of graph.cpp:332-347: for u ascending, for uu in sorted nbrs_[u], u < uu.
    for (uint32_t u = 0; u < nv; u++)
        for (auto &p : q.nbrs[u]) {
            if (u > p.first) continue;
            int idx = (int)q.qe_list.size();
            q.qe_list.emplace_back(u, p.first);
            q.qe_elabel.push_back(p.second);
            q.qe_index[u * nv + p.first] = idx;
            q.qe_index[p.first * nv + u] = idx;
        }
    // Connectivity: every matching order of plan.cpp grows from the updated edge.
    std::vector<int> seen(nv, 0);
    std::vector<uint32_t> stack{0};
    seen[0] = 1;
    while (!stack.empty()) {
        uint32_t u = stack.back();
        stack.pop_back();
        for (auto &p : q.nbrs[u])
            if (!seen[p.first]) {
                seen[p.first] = 1;
                stack.push_back(p.first);
            }
    }
    for (uint32_t u = 0; u < nv; u++)
        if (!seen[u]) return "the query graph must be connected";
    // NLF groups (graph.cpp:295-330): neighbours grouped by (edge label, neighbour label).
    q.nlf.assign(nv, {});
    for (uint32_t u = 0; u < nv; u++) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> groups;
        for (auto &p : q.nbrs[u]) groups[{p.second, q.vlabel[p.first]}]++;
        for (auto &g : groups) q.nlf[u].push_back({g.first.first, g.first.second, g.second});
    }
    return "";
}

}  // namespace csm
