#include "plan.h"

#include <algorithm>
#include <cstring>
#include <limits>
#include <map>
#include <sstream>

namespace csm {

namespace {

float avg_of(const Query &q, const EdgeStats &st, uint32_t u, uint32_t uu) { return st.avg[u * q.nv + uu]; }

// Rules 0-4 of the GAMMA / GCSM-v2 vertex selection (plan.cpp:537-760 and 1866-2080):
// 0 keep extendable vertices whose smallest backward relation average degree is not 1024x
//   larger than the previous one, 1 most backward neighbours, 2 most matched vertices
//   adjacent to its unmatched neighbours, 3 most dangling neighbours, 4 smallest average degree.
uint32_t select_by_gamma_rules(const Query &q, const EdgeStats &st, const std::vector<char> &visited) {
    const uint32_t n = q.nv;
    std::vector<uint32_t> selected, further;
    {
        // The reference stores the average degree in a uint32_t (pair<uint8_t, uint32_t>).
        std::vector<std::pair<uint8_t, uint32_t>> cand;
        for (uint32_t u = 0; u < n; u++) {
            if (visited[u]) continue;
            for (auto &p : q.nbrs[u]) {
                uint32_t bn = p.first;
                if (!visited[bn]) continue;
                uint32_t a = (uint32_t)avg_of(q, st, bn, u);
                if (cand.empty() || cand.back().first != u) cand.emplace_back((uint8_t)u, a);
                else if (avg_of(q, st, bn, u) < (float)cand.back().second) cand.back().second = a;
            }
        }
        std::sort(cand.begin(), cand.end(), [](const auto &a, const auto &b) { return a.second < b.second; });
        size_t new_end = cand.size();
        for (size_t j = 0; j + 1 < cand.size(); j++)
            if (cand[j + 1].second >= cand[j].second * (2u << 9)) {
                new_end = j + 1;
                break;
            }
        for (size_t j = 0; j < new_end; j++) selected.push_back(cand[j].first);
        std::sort(selected.begin(), selected.end());
    }
    auto keep_best = [&](auto score, bool maximize) {
        if (selected.size() <= 1) return;
        further.clear();
        bool first = true;
        double best = 0;
        for (uint32_t u : selected) {
            double s = score(u);
            if (first || (maximize ? s > best : s < best)) {
                best = s;
                first = false;
                further.clear();
                further.push_back(u);
            } else if (s == best) {
                further.push_back(u);
            }
        }
        selected.swap(further);
    };
    // Rule 1 (plan.cpp:597-622).
    keep_best([&](uint32_t u) {
        uint32_t c = 0;
        for (auto &p : q.nbrs[u]) c += visited[p.first] ? 1 : 0;
        return (double)c;
    }, true);
    // Rule 2 (plan.cpp:628-659).
    keep_best([&](uint32_t u) {
        std::vector<char> tv(n, 0);
        uint32_t c = 0;
        for (auto &p : q.nbrs[u]) {
            if (visited[p.first]) continue;
            for (auto &pp : q.nbrs[p.first])
                if (visited[pp.first] && !tv[pp.first]) {
                    tv[pp.first] = 1;
                    c++;
                }
        }
        return (double)c;
    }, true);
    // Rule 3 (plan.cpp:667-702).
    keep_best([&](uint32_t u) {
        uint32_t c = 0;
        for (auto &p : q.nbrs[u]) {
            if (visited[p.first]) continue;
            bool dangling = true;
            for (auto &pp : q.nbrs[p.first])
                if (visited[pp.first]) {
                    dangling = false;
                    break;
                }
            c += dangling ? 1 : 0;
        }
        return (double)c;
    }, true);
    // Rule 4 (plan.cpp:709-737).
    keep_best([&](uint32_t u) {
        float m = std::numeric_limits<float>::max();
        for (auto &p : q.nbrs[u])
            if (visited[p.first]) m = std::min(m, avg_of(q, st, p.first, u));
        return (double)m;
    }, false);
    return selected[0];
}

std::vector<uint8_t> gamma_like_order(const Query &q, const EdgeStats &st, uint32_t a, uint32_t b) {
    std::vector<char> visited(q.nv, 0);
    std::vector<uint8_t> order{(uint8_t)a, (uint8_t)b};
    visited[a] = visited[b] = 1;
    while (order.size() < q.nv) {
        uint32_t u = select_by_gamma_rules(q, st, visited);
        order.push_back((uint8_t)u);
        visited[u] = 1;
    }
    return order;
}

// Starting edge of the GCSM v2 order (plan.cpp:396-534).
std::pair<uint32_t, uint32_t> gcsm_start_edge(const Query &q, const EdgeStats &st, uint32_t u0, uint32_t u1) {
    std::vector<std::pair<uint32_t, uint32_t>> sel, fur;
    size_t best = 0;
    for (auto &e : q.qe_list) {
        size_t s = q.nbrs[e.first].size() + q.nbrs[e.second].size();
        if (s > best) {
            best = s;
            sel.clear();
            sel.push_back(e);
        } else if (s == best) {
            sel.push_back(e);
        }
    }
    if (sel.size() > 1) {  // most triangles
        uint32_t bt = 0;
        fur.clear();
        for (auto &e : sel) {
            uint32_t t = 0;
            for (uint32_t w = 0; w < q.nv; w++) t += (q.adjacent(w, e.first) && q.adjacent(w, e.second)) ? 1 : 0;
            if (t > bt) {
                bt = t;
                fur.clear();
                fur.push_back(e);
            } else if (t == bt) {
                fur.push_back(e);
            }
        }
        sel.swap(fur);
    }
    if (sel.size() > 1) {  // prefer the updated edge
        for (auto &e : sel)
            if ((e.first == u0 && e.second == u1) || (e.first == u1 && e.second == u0)) {
                sel.assign(1, {u0, u1});
                break;
            }
    }
    if (sel.size() > 1) {  // fewest candidate edges
        uint32_t bc = UINT32_MAX;
        fur.clear();
        for (auto &e : sel) {
            uint32_t c = st.card[e.first * q.nv + e.second];
            if (c < bc) {
                bc = c;
                fur.clear();
                fur.push_back(e);
            } else if (c == bc) {
                fur.push_back(e);
            }
        }
        sel.swap(fur);
    }
    if (sel.size() > 1) {  // smallest sum of neighbouring average degrees
        float bs = std::numeric_limits<float>::max();
        fur.clear();
        for (auto &e : sel) {
            float s = 0.f;
            for (auto &p : q.nbrs[e.first])
                if (p.first != e.second) s += avg_of(q, st, e.first, p.first);
            for (auto &p : q.nbrs[e.second])
                if (p.first != e.first) s += avg_of(q, st, e.second, p.first);
            if (s < bs) {
                bs = s;
                fur.clear();
                fur.push_back(e);
            } else if (s == bs) {
                fur.push_back(e);
            }
        }
        sel.swap(fur);
    }
    return sel[0];
}

// RI order (plan.cpp:195-368): start at the first vertex of maximum degree, then rules 1-3
// over all unmatched vertices.
std::vector<uint8_t> ri_priority(const Query &q) {
    const uint32_t n = q.nv;
    std::vector<char> visited(n, 0);
    std::vector<uint8_t> order;
    uint32_t best = 0, start = 0;
    for (uint32_t u = 0; u < n; u++)
        if (q.degree(u) > best) {
            best = q.degree(u);
            start = u;
        }
    order.push_back((uint8_t)start);
    visited[start] = 1;
    for (uint32_t step = 1; step < n; step++) {
        std::vector<uint32_t> sel, fur;
        uint32_t bnb = 0;
        for (uint32_t u = 0; u < n; u++) {
            if (visited[u]) continue;
            uint32_t c = 0;
            for (auto &p : q.nbrs[u]) c += visited[p.first] ? 1 : 0;
            if (c > bnb) {
                bnb = c;
                sel.clear();
                sel.push_back(u);
            } else if (c == bnb) {
                sel.push_back(u);
            }
        }
        if (sel.size() > 1) {
            uint32_t bv = 0;
            for (uint32_t u : sel) {
                std::vector<char> tv(n, 0);
                uint32_t c = 0;
                for (auto &p : q.nbrs[u]) {
                    if (visited[p.first]) continue;
                    for (auto &pp : q.nbrs[p.first])
                        if (visited[pp.first] && !tv[pp.first]) {
                            tv[pp.first] = 1;
                            c++;
                        }
                }
                if (c > bv) {
                    bv = c;
                    fur.clear();
                    fur.push_back(u);
                } else if (c == bv) {
                    fur.push_back(u);
                }
            }
            sel.swap(fur);
            fur.clear();
        }
        if (sel.size() > 1) {
            uint32_t bf = 0;
            for (uint32_t u : sel) {
                uint32_t c = 0;
                for (auto &p : q.nbrs[u]) {
                    if (visited[p.first]) continue;
                    bool dangling = true;
                    for (auto &pp : q.nbrs[p.first])
                        if (visited[pp.first]) {
                            dangling = false;
                            break;
                        }
                    c += dangling ? 1 : 0;
                }
                if (c > bf) {
                    bf = c;
                    fur.clear();
                    fur.push_back(u);
                } else if (c == bf) {
                    fur.push_back(u);
                }
            }
            sel.swap(fur);
        }
        order.push_back((uint8_t)sel[0]);
        visited[sel[0]] = 1;
    }
    return order;
}

// Re-anchors a vertex priority list at the updated edge (u0, u1): repeatedly takes the
// first vertex of `prio` that is unmatched and adjacent to a matched one.
std::vector<uint8_t> reanchor(const Query &q, const std::vector<uint8_t> &prio, uint32_t u0, uint32_t u1) {
    std::vector<char> visited(q.nv, 0);
    std::vector<uint8_t> order{(uint8_t)u0, (uint8_t)u1};
    visited[u0] = visited[u1] = 1;
    while (order.size() < q.nv) {
        for (uint8_t u : prio) {
            if (visited[u]) continue;
            bool ext = false;
            for (auto &p : q.nbrs[u]) ext |= visited[p.first] != 0;
            if (!ext) continue;
            order.push_back(u);
            visited[u] = 1;
            break;
        }
    }
    return order;
}

int64_t signed_coef(int block) {  // (-1)^(b-1) (b-1)!
    int64_t f = 1;
    for (int k = 2; k < block; k++) f *= k;
    return (block % 2 == 1) ? f : -f;
}

// Enumerates the set partitions of m items as restricted growth strings a[0..m-1]
// (a[0] = 0, a[i] <= 1 + max(a[0..i-1])); a[i] is the block of item i.
void partitions_from(int i, int maxv, std::vector<int> &a, const std::function<void(const std::vector<int> &)> &fn) {
    if (i == (int)a.size()) {
        fn(a);
        return;
    }
    for (int v = 0; v <= maxv + 1; v++) {
        a[i] = v;
        partitions_from(i + 1, std::max(maxv, v), a, fn);
    }
}

void for_each_partition(int m, const std::function<void(const std::vector<int> &)> &fn) {
    std::vector<int> a(m, 0);
    partitions_from(1, 0, a, fn);
}

// Builds the tail bookkeeping for the vertices at depths [tail_start, n).  They are pairwise
// non-adjacent and every neighbour of theirs is matched before tail_start, so each one's
// candidates are the intersection of its backward-neighbour lists (its keys), and the number of
// injective assignments is a polynomial in intersection sizes.  Returns false when the tail
// exceeds the device limits (the caller then shortens it).
bool build_tail(const Query &q, const HostPlan &hp, int qe, const RelOf &rel_of, DevTail &tail,
                std::vector<DevTailTerm> &terms) {
    const int n = (int)hp.order.size();
    std::memset(&tail, 0, sizeof(tail));
    terms.clear();
    if (hp.tail_start >= n) return true;
    struct Leaf {
        uint16_t keys;  // bit k: key k is one of the vertex's lists
        uint32_t label;
    };
    std::vector<Leaf> leaves;
    std::vector<std::tuple<int, int, int>> keys;  // (parent depth, rel, old)
    for (int d = hp.tail_start; d < n; d++) {
        const uint32_t u = hp.order[d];
        Leaf leaf{0, q.vlabel[u]};
        for (uint8_t p : hp.bn[d]) {
            if ((int)p >= hp.tail_start) return false;  // not a tail: a neighbour in the tail
            uint32_t pu = hp.order[p];
            int rel = rel_of(pu, u);
            int old = q.qe_index[pu * q.nv + u] > qe ? 1 : 0;
            auto k = std::make_tuple((int)p, rel, old);
            int ki = (int)(std::find(keys.begin(), keys.end(), k) - keys.begin());
            if (ki == (int)keys.size()) keys.push_back(k);
            if (ki >= CSM_TAIL_MAXKEYS) return false;
            leaf.keys |= (uint16_t)(1u << ki);
        }
        leaves.push_back(leaf);
    }
    if (keys.size() > CSM_TAIL_MAXKEYS) return false;
    tail.nkeys = (uint8_t)keys.size();
    for (size_t k = 0; k < keys.size(); k++) {
        tail.key_parent[k] = (uint8_t)std::get<0>(keys[k]);
        tail.key_rel[k] = (uint16_t)std::get<1>(keys[k]);
        tail.key_old[k] = (uint8_t)std::get<2>(keys[k]);
        // A key's relation fixes its leaves' label.
        uint32_t leaf_label = 0;
        for (auto &l : leaves)
            if ((l.keys >> k) & 1u) leaf_label = l.label;
        uint16_t excl = 0;
        for (int d = 0; d < n; d++)
            if (q.vlabel[hp.order[d]] == leaf_label) excl |= (uint16_t)(1u << d);
        tail.key_excl[k] = excl;
    }
    std::map<uint32_t, std::vector<uint16_t>> classes;  // label -> the key sets of its vertices
    for (auto &l : leaves) classes[l.label].push_back(l.keys);
    if (classes.size() > CSM_TAIL_MAXCLASSES) return false;
    std::vector<uint16_t> masks;
    auto mask_id = [&](uint16_t m) -> int {
        auto it = std::find(masks.begin(), masks.end(), m);
        if (it != masks.end()) return (int)(it - masks.begin());
        masks.push_back(m);
        return (int)masks.size() - 1;
    };
    int c = 0;
    for (auto &cl : classes) {
        const std::vector<uint16_t> &ks = cl.second;
        const int m = (int)ks.size();
        if (m > 7) return false;
        tail.class_term_begin[c] = (uint16_t)terms.size();
        // Inclusion-exclusion over set partitions: the number of injective assignments of
        // the class's leaves is sum over partitions pi of prod_B (-1)^{|B|-1}(|B|-1)! |cap_B|.
        std::map<std::vector<int>, int64_t> acc;
        bool ok = true;
        for_each_partition(m, [&](const std::vector<int> &a) {
            int nb = 0;
            for (int x : a) nb = std::max(nb, x + 1);
            std::vector<uint16_t> bm(nb, 0);
            std::vector<int> bs(nb, 0);
            for (int i = 0; i < m; i++) {
                bm[a[i]] |= ks[i];  // a block's vertices share one candidate: all their lists
                bs[a[i]]++;
            }
            int64_t coef = 1;
            std::vector<int> f;
            for (int b = 0; b < nb; b++) {
                coef *= signed_coef(bs[b]);
                int id = mask_id(bm[b]);
                if (id >= CSM_TAIL_MAXMASKS) ok = false;
                f.push_back(id);
            }
            std::sort(f.begin(), f.end());
            acc[f] += coef;
        });
        if (!ok) return false;
        for (auto &t : acc) {
            if (t.second == 0) continue;
            DevTailTerm term{};
            term.coef = t.second;
            term.nf = (uint8_t)t.first.size();
            for (size_t j = 0; j < t.first.size(); j++) term.f[j] = (uint8_t)t.first[j];
            terms.push_back(term);
        }
        c++;
    }
    tail.nclasses = (uint8_t)c;
    tail.class_term_begin[c] = (uint16_t)terms.size();
    if (masks.size() > CSM_TAIL_MAXMASKS) return false;
    tail.nmasks = (uint8_t)masks.size();
    tail.lane_par = 1;
    for (size_t k = 0; k < masks.size(); k++) {
        tail.mask[k] = masks[k];
        if (__builtin_popcount(masks[k]) != 1) tail.lane_par = 0;
    }
    return true;
}

}  // namespace

std::vector<uint8_t> indexing_order(const Query &q, uint32_t u0, uint32_t u1) {
    // BFS from (u0, u1), neighbours in sorted order (plan.cpp:1548-1577).
    std::vector<uint8_t> order{(uint8_t)u0, (uint8_t)u1};
    std::vector<char> visited(q.nv, 0);
    visited[u0] = visited[u1] = 1;
    std::vector<uint32_t> level{u0, u1}, next;
    while (!level.empty()) {
        next.clear();
        for (uint32_t v : level)
            for (auto &p : q.nbrs[v])
                if (!visited[p.first]) {
                    visited[p.first] = 1;
                    next.push_back(p.first);
                    order.push_back((uint8_t)p.first);
                }
        level.swap(next);
    }
    return order;
}

std::vector<HostPlan> build_plans(const Query &q, uint16_t query_id, uint32_t nlf_base,
                                  const EdgeStats &st, const PlanOptions &opt, const RelOf &rel_of) {
    std::vector<HostPlan> plans;
    const uint32_t n = q.nv;
    for (uint32_t i = 0; i < q.qe_list.size(); i++) {
        const uint32_t u0 = q.qe_list[i].first, u1 = q.qe_list[i].second;
        std::vector<uint8_t> order;
        switch (opt.order) {
            case Order::kIndexing: order = indexing_order(q, u0, u1); break;
            case Order::kGamma: order = gamma_like_order(q, st, u0, u1); break;
            case Order::kGcsm: {
                auto se = gcsm_start_edge(q, st, u0, u1);
                // Orientation by the indexing order (plan.cpp:517-534).
                auto io = indexing_order(q, u0, u1);
                uint32_t a = se.first, b = se.second;
                for (uint8_t v : io) {
                    if (v == se.first) break;
                    if (v == se.second) {
                        std::swap(a, b);
                        break;
                    }
                }
                order = reanchor(q, gamma_like_order(q, st, a, b), u0, u1);
                break;
            }
            case Order::kRi: order = reanchor(q, ri_priority(q), u0, u1); break;
        }
        HostPlan hp;
        // Cartesian tail: query leaves after the starting edge move to the end of the order
        // (they constrain nothing else), and depth >= tail_start is counted arithmetically.
        // The tail then grows backwards over every last head vertex adjacent to no tail vertex:
        // its neighbours are all matched before it, so given the head it is independent of the
        // other tail vertices too, and its candidates are an intersection of head lists.
        int tail_start = (int)n;
        if (opt.cartesian && !opt.materialize && n > 2) {
            std::vector<uint8_t> head(order.begin(), order.begin() + 2), leaves;
            for (size_t d = 2; d < n; d++) (q.degree(order[d]) == 1 ? leaves : head).push_back(order[d]);
            tail_start = (int)head.size();
            head.insert(head.end(), leaves.begin(), leaves.end());
            order = head;
            const int leaf_start = tail_start;
            while (tail_start > 2) {
                bool free_vertex = true;
                for (uint32_t t = (uint32_t)tail_start; t < n; t++)
                    if (q.adjacent(order[tail_start - 1], order[t])) free_vertex = false;
                if (!free_vertex) break;
                tail_start--;
            }
            // Without leaves, one or two such vertices are counted faster by the last-level
            // loops (the shared last level covers two).
            if (leaf_start == (int)n && (int)n - tail_start < 3) tail_start = (int)n;
        }
        hp.order = order;
        hp.bn.assign(n, {});
        for (uint32_t d = 1; d < n; d++) {
            for (uint32_t k = 0; k < d; k++)
                if (q.adjacent(order[k], order[d])) hp.bn[d].push_back((uint8_t)k);
            const uint32_t u = order[d];
            std::sort(hp.bn[d].begin(), hp.bn[d].end(), [&](uint8_t a, uint8_t b) {
                return st.avg[order[a] * n + u] < st.avg[order[b] * n + u];
            });
        }
        // Shorten the tail until its bookkeeping fits the device tables.
        DevTail tail{};
        std::vector<DevTailTerm> terms;
        hp.tail_start = tail_start;
        while (hp.tail_start < (int)n && !build_tail(q, hp, (int)i, rel_of, tail, terms)) hp.tail_start++;
        if (hp.tail_start >= (int)n) {
            hp.tail_start = (int)n;
            std::memset(&tail, 0, sizeof(tail));
            terms.clear();
        }
        hp.terms = terms;
        DevPlan &dp = hp.dev;
        std::memset(&dp, 0, sizeof(dp));
        dp.query = query_id;
        dp.n = (uint8_t)n;
        dp.qe = (uint8_t)i;
        dp.tail_start = (uint8_t)hp.tail_start;
        dp.materialize = opt.materialize ? 1 : 0;
        dp.seed_rel = rel_of(order[0], order[1]);
        for (uint32_t d = 0; d < n; d++) dp.order[d] = order[d];
        dp.nlf0 = nlf_base + order[0];
        dp.nlf1 = nlf_base + order[1];
        uint32_t bn_base = 0;
        for (uint32_t d = 0; d < n; d++) {
            DevLevel &lv = dp.lv[d];
            lv.bn_base = (uint8_t)bn_base;
            bn_base += (uint32_t)hp.bn[d].size();
            lv.qv = order[d];
            lv.nbn = (uint8_t)hp.bn[d].size();
            // All query neighbours matched before this level: the NLF filter is implied.
            lv.nlf_bitmap = hp.bn[d].size() == q.nbrs[order[d]].size() ? CSM_NO_BITMAP : nlf_base + order[d];
            for (uint32_t j = 0; j < d; j++)
                if (q.vlabel[order[j]] == q.vlabel[order[d]]) lv.excl_mask |= (uint16_t)(1u << j);
            for (size_t k = 0; k < hp.bn[d].size(); k++) {
                uint32_t bu = order[hp.bn[d][k]];
                lv.bn_depth[k] = hp.bn[d][k];
                lv.bn_rel[k] = rel_of(bu, order[d]);
                if (q.qe_index[bu * n + order[d]] > (int)i) lv.old_mask |= (uint16_t)(1u << k);
            }
        }
        dp.tail = tail;
        dp.nterms = (uint32_t)terms.size();
        if (hp.tail_start == (int)n && n >= 4) {
            dp.shared_last = 1;
            for (uint8_t b : hp.bn[n - 1])
                if (b == n - 2) dp.shared_last = 0;
        }
        dp.expand_stop = (uint8_t)(dp.shared_last ? n - 2 : hp.tail_start - 1);
        dp.memo_slot = CSM_NO_MEMO;
        const int c = hp.tail_start - 1;
        if (hp.tail_start < (int)n && tail.lane_par && c >= 3 && hp.bn[c].size() == 1 && dp.lv[c].excl_mask == 0) {
            bool pendant = true;
            for (int k = 0; k < tail.nkeys; k++)
                if (tail.key_parent[k] != c || (tail.key_excl[k] & ((1u << c) - 1u)) != 0) pendant = false;
            if (pendant) {
                dp.memo_slot = CSM_MEMO_PENDING;
                dp.memo_depth = hp.bn[c][0];
                dp.expand_stop = (uint8_t)(c - 1);
            }
        }
        plans.push_back(hp);
    }
    return plans;
}

std::string describe_plans(const Query &q, const std::vector<HostPlan> &plans) {
    std::ostringstream os;
    os << "Orders:\n";
    for (size_t i = 0; i < plans.size(); i++) {
        const HostPlan &hp = plans[i];
        os << '[' << q.qe_list[i].first << ',' << q.qe_list[i].second << "]:\n    order: ";
        for (size_t d = 0; d < hp.order.size(); d++) {
            os << (uint32_t)hp.order[d] << "-(";
            for (size_t k = 0; k < hp.bn[d].size(); k++) {
                os << (uint32_t)hp.order[hp.bn[d][k]] << '@' << (uint32_t)hp.bn[d][k];
                if (hp.dev.lv[d].old_mask & (1u << k)) os << "*";
                if (k + 1 < hp.bn[d].size()) os << ' ';
            }
            os << ") ";
        }
        os << "\n    tail: " << (hp.tail_start < (int)hp.order.size() ? "from depth " + std::to_string(hp.tail_start) : std::string("none"))
           << ", " << hp.terms.size() << " terms" << (hp.dev.shared_last ? ", last level shared by the level above" : "")
           << (hp.dev.memo_slot != CSM_NO_MEMO ? ", pendant counting level" : "")
           << "\n";
    }
    return os.str();
}

}  // namespace csm
