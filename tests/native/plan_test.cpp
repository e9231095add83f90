// Host-only checks of the planner (gcsm-bu_b200/csrc/plan.cpp) on random labelled queries:
//  - every order is a permutation that starts with the updated query edge's endpoints;
//  - the backward neighbours of each depth are exactly the query neighbours matched earlier,
//    so every query edge is checked once;
//  - every neighbour of a tail vertex is matched before the tail (leaves, and the vertices the
//    tail grows over);
//  - the tail's inclusion-exclusion polynomial, evaluated the way the enumeration kernel does,
//    equals a brute-force count of injective tail assignments on random candidate lists (a tail
//    vertex's candidates: the intersection of its lists).
#include <cstdio>
#include <cstring>
#include <map>
#include <random>
#include <set>
#include <tuple>
#include <vector>

#include "plan.h"
#include "query.h"

using namespace csm;

namespace {

int fail(const char *what, int qn, int plan) {
    std::printf("FAIL %s (query %d, plan %d)\n", what, qn, plan);
    return 1;
}

bool in_list(const std::vector<int> &l, int x) {
    for (int y : l)
        if (y == x) return true;
    return false;
}

// Brute force: number of maps tail vertex -> element of all its lists, injective within each
// label class.
uint64_t brute(const std::vector<std::vector<int>> &lists, int universe, const std::vector<uint16_t> &leaf_keys,
               const std::vector<uint32_t> &leaf_label, size_t i, std::vector<int> &chosen) {
    if (i == leaf_keys.size()) return 1;
    uint64_t total = 0;
    for (int x = 0; x < universe; x++) {
        bool cand = true;
        for (size_t k = 0; k < lists.size(); k++)
            if (((leaf_keys[i] >> k) & 1u) && !in_list(lists[k], x)) cand = false;
        if (!cand) continue;
        bool clash = false;
        for (size_t j = 0; j < i; j++)
            if (leaf_label[j] == leaf_label[i] && chosen[j] == x) clash = true;
        if (clash) continue;
        chosen[i] = x;
        total += brute(lists, universe, leaf_keys, leaf_label, i + 1, chosen);
    }
    return total;
}

}  // namespace

int main() {
    std::mt19937 rng(2024);
    int checked_tails = 0;
    for (int qn = 0; qn < 400; qn++) {
        // Random connected query: a random tree plus a few extra edges, 3..9 vertices, labels
        // from a small alphabet so that leaves often share labels.
        const uint32_t nv = 3 + rng() % 7;
        std::vector<uint32_t> vl(nv), src, dst, el;
        for (auto &x : vl) x = rng() % 3;
        std::set<std::pair<uint32_t, uint32_t>> seen;
        for (uint32_t v = 1; v < nv; v++) {
            const uint32_t p = rng() % v;
            src.push_back(p);
            dst.push_back(v);
            el.push_back(rng() % 2);
            seen.insert({p, v});
        }
        const int extra = (int)(rng() % 3);
        for (int e = 0; e < extra; e++) {
            uint32_t a = rng() % nv, b = rng() % nv;
            if (a == b) continue;
            if (a > b) std::swap(a, b);
            if (!seen.insert({a, b}).second) continue;
            src.push_back(a);
            dst.push_back(b);
            el.push_back(rng() % 2);
        }
        Query q;
        const std::string err = build_query(nv, vl.data(), (uint32_t)src.size(), src.data(), dst.data(), el.data(), q);
        if (!err.empty()) return std::printf("build_query: %s\n", err.c_str()), 1;
        std::map<std::tuple<uint32_t, uint32_t, uint32_t>, uint16_t> rels;
        RelOf rel_of = [&](uint32_t u, uint32_t uu) -> uint16_t {
            auto k = std::make_tuple(q.vlabel[u], q.edge_label(u, uu), q.vlabel[uu]);
            auto it = rels.find(k);
            if (it != rels.end()) return it->second;
            const uint16_t id = (uint16_t)rels.size();
            rels[k] = id;
            return id;
        };
        EdgeStats st;
        st.card.assign(nv * nv, 0);
        st.avg.assign(nv * nv, 0.f);
        for (uint32_t u = 0; u < nv; u++)
            for (auto &p : q.nbrs[u]) {
                st.card[u * nv + p.first] = 1 + rng() % 1000;
                st.avg[u * nv + p.first] = 1.f + (float)(rng() % 100);
            }
        for (int order = 0; order < 4; order++) {
            PlanOptions po;
            po.order = (Order)order;
            po.cartesian = true;
            const std::vector<HostPlan> plans = build_plans(q, 0, 0, st, po, rel_of);
            if (plans.size() != q.qe_list.size()) return fail("plan count", qn, -1);
            for (size_t pi = 0; pi < plans.size(); pi++) {
                const HostPlan &hp = plans[pi];
                const uint32_t n = (uint32_t)hp.order.size();
                if (n != nv) return fail("order length", qn, (int)pi);
                std::vector<int> depth(nv, -1);
                for (uint32_t d = 0; d < n; d++) {
                    if (hp.order[d] >= nv || depth[hp.order[d]] >= 0) return fail("not a permutation", qn, (int)pi);
                    depth[hp.order[d]] = (int)d;
                }
                const auto &qe = q.qe_list[pi];
                if (!((hp.order[0] == qe.first && hp.order[1] == qe.second) ||
                      (hp.order[0] == qe.second && hp.order[1] == qe.first)))
                    return fail("order does not start at the updated edge", qn, (int)pi);
                for (uint32_t d = 1; d < n; d++) {
                    std::set<int> want, got;
                    for (auto &p : q.nbrs[hp.order[d]])
                        if (depth[p.first] < (int)d) want.insert(depth[p.first]);
                    for (uint8_t b : hp.bn[d]) got.insert(b);
                    if (d == 1) want.erase(0), got.erase(0);  // the seed edge itself
                    if (want != got) return fail("backward neighbours", qn, (int)pi);
                    if (want.empty() && d > 1) return fail("disconnected prefix", qn, (int)pi);
                    if (d < 2) continue;
                    // Injectivity is checked against the same-label prefix depths only, and the
                    // NLF filter is dropped exactly where every query neighbour is backward.
                    const DevLevel &lv = hp.dev.lv[d];
                    for (uint32_t j = 0; j < n; j++) {
                        const bool same = j < d && q.vlabel[hp.order[j]] == q.vlabel[hp.order[d]];
                        if (same != (((lv.excl_mask >> j) & 1u) != 0)) return fail("level exclusion depths", qn, (int)pi);
                    }
                    const bool all_back = hp.bn[d].size() == q.nbrs[hp.order[d]].size();
                    if (all_back != (lv.nlf_bitmap == CSM_NO_BITMAP)) return fail("implied NLF filter", qn, (int)pi);
                }
                const int ts = hp.tail_start;
                // The last level is shared by the candidates of level n - 2 exactly when it has
                // no backward neighbour there (and no tail follows); expansion then stops at n - 2.
                bool shared = ts == (int)n && n >= 4;
                for (uint8_t b : hp.bn[n - 1])
                    if (b == n - 2) shared = false;
                if ((hp.dev.shared_last != 0) != shared) return fail("shared last level", qn, (int)pi);
                // Pendant counting level c = ts - 1: one backward neighbour, every tail vertex
                // hangs off c alone, single-list tail terms, and no vertex before c shares a label
                // with c or with a tail vertex.
                const int c = ts - 1;
                bool pendant = ts < (int)n && c >= 3 && hp.bn[c].size() == 1 && hp.dev.tail.lane_par;
                for (uint32_t d = (uint32_t)ts; pendant && d < n; d++)
                    if (hp.bn[d].size() != 1 || hp.bn[d][0] != c) pendant = false;
                for (int j = 0; pendant && j < c; j++)
                    for (uint32_t d = (uint32_t)c; d < n; d++)
                        if (q.vlabel[hp.order[j]] == q.vlabel[hp.order[d]]) pendant = false;
                if ((hp.dev.memo_slot == CSM_MEMO_PENDING) != pendant) return fail("pendant counting level", qn, (int)pi);
                if (pendant && hp.dev.memo_depth != hp.bn[c][0]) return fail("pendant table depth", qn, (int)pi);
                if (hp.dev.expand_stop != (shared ? n - 2 : pendant ? (uint32_t)c - 1 : (uint32_t)ts - 1))
                    return fail("expansion stop", qn, (int)pi);
                for (uint32_t d = (uint32_t)ts; d < n; d++) {
                    if (hp.bn[d].size() != q.nbrs[hp.order[d]].size()) return fail("tail neighbour after the tail", qn, (int)pi);
                    for (uint8_t b : hp.bn[d])
                        if ((int)b >= ts) return fail("tail neighbour inside the tail", qn, (int)pi);
                }
                if (ts >= (int)n) continue;
                // Evaluate the tail polynomial as the kernel does, on random candidate lists.
                const DevTail &T = hp.dev.tail;
                std::vector<uint16_t> leaf_keys;
                std::vector<uint32_t> leaf_label;
                for (uint32_t d = (uint32_t)ts; d < n; d++) {
                    const uint32_t u = hp.order[d];
                    uint16_t keys = 0;
                    for (uint8_t p : hp.bn[d]) {
                        const uint32_t pu = hp.order[p];
                        const int rel = rel_of(pu, u);
                        const int old = q.qe_index[pu * nv + u] > (int)pi ? 1 : 0;
                        int key = -1;
                        for (int k = 0; k < T.nkeys; k++)
                            if (T.key_parent[k] == p && T.key_rel[k] == rel && T.key_old[k] == old) key = k;
                        if (key < 0) return fail("tail vertex without a tail key", qn, (int)pi);
                        for (uint32_t j = 0; j < n; j++) {
                            const bool same = q.vlabel[hp.order[j]] == q.vlabel[u];
                            if (same != (((T.key_excl[key] >> j) & 1u) != 0)) return fail("exclusion depths", qn, (int)pi);
                        }
                        keys |= (uint16_t)(1u << key);
                    }
                    leaf_keys.push_back(keys);
                    leaf_label.push_back(q.vlabel[u]);
                }
                for (int trial = 0; trial < 20; trial++) {
                    const int universe = 3 + (int)(rng() % 6);
                    std::vector<std::vector<int>> lists(T.nkeys);
                    for (auto &l : lists)
                        for (int x = 0; x < universe; x++)
                            if (rng() % 2) l.push_back(x);
                    unsigned long long total = 1;
                    for (int c = 0; c < T.nclasses; c++) {
                        long long s = 0;
                        for (int t = T.class_term_begin[c]; t < T.class_term_begin[c + 1]; t++) {
                            long long prod = hp.terms[t].coef;
                            for (int j = 0; j < hp.terms[t].nf; j++) {
                                const uint16_t mk = T.mask[hp.terms[t].f[j]];
                                // |intersection of the lists in the mask|
                                long long cnt = 0;
                                for (int x = 0; x < universe; x++) {
                                    bool all = true;
                                    for (int k = 0; k < T.nkeys; k++)
                                        if ((mk >> k) & 1u) {
                                            bool in = false;
                                            for (int y : lists[k]) in |= (y == x);
                                            all &= in;
                                        }
                                    cnt += all;
                                }
                                prod *= cnt;
                            }
                            s += prod;
                        }
                        total *= (unsigned long long)s;
                    }
                    std::vector<int> chosen(leaf_keys.size());
                    const uint64_t want = brute(lists, universe, leaf_keys, leaf_label, 0, chosen);
                    if (total != want) {
                        std::printf("tail count %llu, brute force %llu\n", total, (unsigned long long)want);
                        return fail("tail polynomial", qn, (int)pi);
                    }
                }
                checked_tails++;
            }
        }
    }
    if (checked_tails < 100) return std::printf("too few tails checked: %d\n", checked_tails), 1;
    std::printf("ok %d\n", checked_tails);
    return 0;
}
