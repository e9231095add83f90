// Persistent warp-DFS enumeration of incremental matches.
//
// Replaces the reference's enumeration kernels: write_initial_partial_results
// (kernels/enumeration.cu:24-79), extendBFSDFSRegTwo (enumeration.cu:407-781),
// gamma_enumerate with its work stealing (kernels/gamma_enumeration.cu:209-880) and the
// Cartesian-product flattening GetNumTree / enumerateCartesianProductTree
// (kernels/cartesian_product.cu:193-284).
//
// One launch covers every (query, updated query edge) plan of a batch.  A warp owns one work
// item at a time and walks its subtree depth first: at each level the candidates are the
// entries of the smallest backward-neighbour list (the pivot), filtered 32 at a time by the
// lanes (flag rule, NLF bitmap, injectivity, membership in the other backward lists by binary
// search) and compacted with ballot/popc into a per-level shared-memory buffer.
//
// Counting rule of the per-query-edge decomposition (technique_permutation.h:125-212): for the
// plan of query edge i the starting edge is a batch edge; an edge matched to a query edge with
// index > i must not be a batch edge; edges of query edges < i may be either.  Every new
// embedding is counted exactly once, at the largest query-edge index it maps to a batch edge.
//
// Load balance: warps first take seed chunks from a ticket counter.  A warp that runs out of
// work posts a request; a busy warp that takes a request splits off part of its pending
// work (the upper half of a candidate range, or buffered sibling candidates) into a global
// queue.  Every wait is bounded; a warp never waits on another warp's progress to finish its
// own items, so exhausting a bound only costs balance, never a result.
//
// Tail leaves (query vertices of degree one matched after their neighbour) are not enumerated:
// their number of injective assignments is computed from list sizes by inclusion-exclusion.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace csm {

namespace {

struct __align__(16) WarpState {
    uint32_t f[CSM_MAXQV];
    uint32_t buf[CSM_MAXQV][CSM_WARP];
    uint32_t lo[CSM_MAXQV];
    uint32_t hi[CSM_MAXQV];
    uint32_t base[CSM_MAXQV];
    // Backward-neighbour lists of every level, in one flat array: level d uses slots
    // [lv[d].bn_base, lv[d].bn_base + nbn) (all levels together hold at most CSM_MAXQE lists).
    uint32_t poff[CSM_MAXQE];
    uint32_t psz[CSM_MAXQE];
    uint32_t cur[CSM_MAXQE];   // per probe list: entries before it are below the next chunk
    uint8_t bnb[CSM_MAXQV];
    uint32_t nlf[CSM_MAXQV];
    uint16_t oldm[CSM_MAXQV];
    uint16_t exm[CSM_MAXQV];   // per level: prefix depths the candidate may coincide with
    uint8_t nbuf[CSM_MAXQV];
    uint8_t pos[CSM_MAXQV];
    uint8_t piv[CSM_MAXQV];
    uint8_t nbn[CSM_MAXQV];
    uint32_t t_off[CSM_TAIL_MAXKEYS];
    uint32_t t_size[CSM_TAIL_MAXKEYS];
    uint32_t t_flag[CSM_TAIL_MAXKEYS];
    uint32_t t_excl[CSM_TAIL_MAXKEYS];
    uint32_t t_cur[CSM_TAIL_MAXKEYS];  // cursor of a probed list while an intersection is counted
    unsigned long long msize[CSM_TAIL_MAXMASKS];
    // Lane-parallel tail: per key whose parent is matched before the counting level, its
    // list and the list size left after the flag rule and the shared prefix.
    uint32_t ts_off[CSM_TAIL_MAXKEYS];
    uint32_t ts_size[CSM_TAIL_MAXKEYS];
    uint32_t ts_base[CSM_TAIL_MAXKEYS];
    uint32_t ts_cur[CSM_TAIL_MAXKEYS];  // cursor of the shared list over ascending candidates
    uint32_t item_plan;
    uint32_t item_depth;
    uint32_t item_lo;
    uint32_t item_hi;
    // Shared last level (DevPlan.shared_last): its candidate count for the current prefix
    // f[0..n-3], and whether it is being counted (1) or known (2).
    unsigned long long sl_count;
    uint32_t sl_state;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t warp_min_index(uint32_t v, uint32_t lane) {
    // Returns the lane holding the smallest v (smallest lane on ties).
    unsigned long long key = ((unsigned long long)v << 5) | lane;
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other < key ? other : key;
    }
    return (uint32_t)(key & 31u);
}

__device__ __forceinline__ const uint32_t *bitmap(const EnumParams &P, uint32_t id) {
    return P.bits + (size_t)id * P.words;
}

// Records the launch's first failed consistency check (the caller skips what failed it).
__device__ void record_bad(const EnumParams &P, uint32_t where, uint32_t a, uint32_t b, uint32_t c) {
    if (atomicCAS(&P.ctrl->bad_where, 0u, where) == 0u) {
        P.ctrl->bad_a = a;
        P.ctrl->bad_b = b;
        P.ctrl->bad_c = c;
    }
    atomicOr(&P.ctrl->error, CSM_ERRBIT_CORRUPT);
}

// {offset, size} of list (rel, v), checked against the vertex range and the pool; a list that
// fails is recorded and read as empty.
__device__ __forceinline__ uint2 list_of(const EnumParams &P, uint32_t rel, uint32_t v, uint32_t level) {
    if (v >= P.g.V || rel >= P.g.R) {
        record_bad(P, CSM_BAD_LIST, v, rel, 0x80000000u | level);
        return make_uint2(0u, 0u);
    }
    const uint2 ms = __ldg(P.g.meta + (size_t)rel * P.g.V + v);
    if ((unsigned long long)ms.x + ms.y > P.g.pool_cap) {
        record_bad(P, CSM_BAD_LIST, ms.x, ms.y, level);
        return make_uint2(0u, 0u);
    }
    return ms;
}

// First index in [lo, hi) of the sorted list L whose entry is >= key2, found by the whole warp
// with 32-ary search: each round reads 32 evenly spaced entries and keeps the bracket that
// holds the answer, so a list of n entries costs about log32(n) dependent reads.
__device__ __forceinline__ uint32_t warp_lower_bound(const uint32_t *L, uint32_t lo, uint32_t hi, uint32_t key2,
                                                     uint32_t lane) {
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t p = lo + (lane + 1) * step - 1;
        const uint32_t v = p < hi ? __ldg(L + p) : 0xFFFFFFFFu;
        const uint32_t c = __popc(__ballot_sync(0xffffffffu, v < key2));
        const uint32_t nhi = lo + (c + 1) * step - 1;
        lo = lo + c * step;
        if (nhi < hi) hi = nhi;
    }
    const uint32_t p = lo + lane;
    const uint32_t v = p < hi ? __ldg(L + p) : 0xFFFFFFFFu;
    return lo + __popc(__ballot_sync(0xffffffffu, v < key2));
}

// Lower bound of key2 among the 32 register-held window entries (sorted, padded with ~0).
__device__ __forceinline__ uint32_t shfl_lower_bound(uint32_t win, uint32_t key2) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1)
        if (__shfl_sync(0xffffffffu, win, pos + step - 1) < key2) pos += step;
    return pos;
}

// Flagged entries of list (rel, x) in this phase (batch edges of that list), 0 if none.
__device__ __forceinline__ uint32_t flagged_in_list(const EnumParams &P, uint32_t rel, uint32_t x) {
    // Lists of vertices no batch key starts from hold no batch entry: skip the key search.
    if (P.touched != nullptr && !((__ldg(P.touched + (x >> 5)) >> (x & 31)) & 1u)) return 0u;
    const unsigned long long lk = P.kl.list_key(rel, x);
    const uint32_t h = find_list_head(P.keys, P.m, P.kl, lk);
    return (h < P.m && P.kl.list_of(__ldg(P.keys + h)) == lk) ? __ldg(P.seg_flagged + h) : 0u;
}

// Lane-parallel tail, shared part: for the counting level d = tail_start - 1 and the current
// prefix f[0..d-1], every tail key whose parent is matched before depth d gets its list and
// the number of its entries the leaves may still use given that prefix.
__device__ void prep_tail_shared(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t d) {
    const uint32_t lane = lane_id();
    const DevTail *T = &pl->tail;
    const uint32_t nkeys = __ldg(&T->nkeys);
    if (lane < nkeys) {
        const uint32_t pd = __ldg(&T->key_parent[lane]);
        if (pd < d) {
            const uint32_t rel = __ldg(&T->key_rel[lane]);
            const bool old = __ldg(&T->key_old[lane]) != 0;
            const uint32_t x = S.f[pd];
            const uint2 ms = list_of(P, rel, x, 100 + d);
            uint32_t left = ms.y - (old ? flagged_in_list(P, rel, x) : 0u);
            const uint32_t excl = __ldg(&T->key_excl[lane]);
            for (uint32_t j = 0; j < d; j++) {
                if (j == pd || !((excl >> j) & 1u)) continue;
                const uint32_t e = find_entry(P.g.pool + ms.x, ms.y, S.f[j]);
                if (e != 0xFFFFFFFFu && !(old && (e & 1u))) left--;
            }
            S.ts_off[lane] = ms.x;
            S.ts_size[lane] = ms.y;
            S.ts_base[lane] = left;
            S.ts_cur[lane] = 0;
        }
    }
    __syncwarp();
}

// Lane-parallel tail, per lane: the tail count of the prefix f[0..d-1] + v, where v is this
// lane's candidate at depth d (for d == 1 the prefix is the seed edge (x0, v)).  Only for
// plans whose masks are single keys (no list intersections).
__device__ unsigned long long tail_count_lane(const uint32_t *ts_base, const uint32_t *f, const EnumParams &P,
                                              const DevPlan *pl,
                                              uint32_t d, uint32_t x0, uint32_t v, uint32_t shared_hit,
                                              uint32_t &probes) {
    const DevTail *T = &pl->tail;
    const uint32_t nkeys = __ldg(&T->nkeys);
    uint32_t ksize[CSM_TAIL_MAXKEYS];
#pragma unroll
    for (uint32_t k = 0; k < CSM_TAIL_MAXKEYS; k++) {
        if (k >= nkeys) break;
        const uint32_t pd = __ldg(&T->key_parent[k]);
        const uint32_t rel = __ldg(&T->key_rel[k]);
        const bool old = __ldg(&T->key_old[k]) != 0;
        uint32_t left;
        if (pd < d && d >= 2) {
            // Shared list: only this lane's candidate may still sit in it (looked up by the
            // warp beforehand, bit k of shared_hit).
            left = ts_base[k] - ((shared_hit >> k) & 1u);
            (void)old;
        } else {
            const uint32_t x = (pd == d) ? v : x0;  // d >= 2: pd == d; d == 1: parent 0 or 1
            const uint2 ms = list_of(P, rel, x, 200 + d);
            left = ms.y - (old ? flagged_in_list(P, rel, x) : 0u);
            const uint32_t excl = __ldg(&T->key_excl[k]);
            for (uint32_t j = 0; j <= d; j++) {
                if (j == pd || !((excl >> j) & 1u)) continue;
                const uint32_t z = (j == d) ? v : (d == 1 ? x0 : f[j]);
                const uint32_t e = find_entry(P.g.pool + ms.x, ms.y, z);
                probes++;
                if (e != 0xFFFFFFFFu && !(old && (e & 1u))) left--;
            }
        }
        ksize[k] = left;
    }
    // Masks are single keys here: mask mi stands for key ffs(mask) - 1.
    unsigned long long total = 1;
    const DevTailTerm *terms = P.terms + pl->term_begin;
    const uint32_t nclasses = __ldg(&T->nclasses);
    for (uint32_t c = 0; c < nclasses; c++) {
        unsigned long long s = 0;
        const uint32_t tb = __ldg(&T->class_term_begin[c]), te = __ldg(&T->class_term_begin[c + 1]);
        for (uint32_t t = tb; t < te; t++) {
            unsigned long long prod = (unsigned long long)__ldg(&terms[t].coef);
            const uint32_t nf = __ldg(&terms[t].nf);
            for (uint32_t j = 0; j < nf; j++) {
                const uint32_t mk = __ldg(&T->mask[__ldg(&terms[t].f[j])]);
                uint32_t sz = 0;
#pragma unroll
                for (uint32_t k = 0; k < CSM_TAIL_MAXKEYS; k++)
                    if (mk == (1u << k)) sz = ksize[k];
                prod *= sz;
            }
            s += prod;
        }
        total *= s;
    }
    return total;
}

// Sets up level d for the current prefix: the backward-neighbour lists and the pivot.
__device__ void enter_level(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t d, uint32_t rlo,
                            uint32_t rhi) {
    const uint32_t lane = lane_id();
    const DevLevel *lv = &pl->lv[d];
    const uint32_t nbn = __ldg(&lv->nbn);
    uint32_t sz = 0xFFFFFFFFu;
    if (lane < nbn) {
        const uint32_t rel = __ldg(&lv->bn_rel[lane]);
        const uint32_t dep = __ldg(&lv->bn_depth[lane]);
        const uint32_t v = S.f[dep];
        const uint2 ms = list_of(P, rel, v, d);
        const uint32_t slot = __ldg(&lv->bn_base) + lane;
        S.poff[slot] = ms.x;
        S.psz[slot] = ms.y;
        S.cur[slot] = 0;
        sz = ms.y;
    }
    const uint32_t piv = warp_min_index(sz, lane);
    __syncwarp();
    if (lane == 0) {
        S.piv[d] = (uint8_t)piv;
        S.nbn[d] = (uint8_t)nbn;
        const uint32_t bb = __ldg(&lv->bn_base);
        S.bnb[d] = (uint8_t)bb;
        S.base[d] = S.poff[bb + piv];
        const uint32_t psize = S.psz[bb + piv];
        S.lo[d] = rlo;
        S.hi[d] = rhi < psize ? rhi : psize;
        S.nbuf[d] = 0;
        S.pos[d] = 0;
        S.oldm[d] = __ldg(&lv->old_mask);
        S.nlf[d] = __ldg(&lv->nlf_bitmap);
        S.exm[d] = __ldg(&lv->excl_mask);
    }
    __syncwarp();
    if (d + 1 == pl->tail_start && pl->tail_start < pl->n && pl->tail.lane_par) prep_tail_shared(S, P, pl, d);
}

// Size of the intersection of the tail lists in `mask` (at least two), each under its flag rule,
// without the prefix vertices f[0..E-1]: the warp scans the smallest list 32 entries at a time.
// A chunk's entries ascend, so every other list keeps a cursor: the 32 entries at the cursor
// are read with one coalesced load and shuffles find each candidate; when the chunk reaches past
// them, a 32-ary warp search brackets the window and lanes search inside it.
__device__ uint32_t tail_intersection(WarpState &S, const EnumParams &P, const DevTail *T, uint32_t nkeys,
                                      uint32_t mask, uint32_t E, uint32_t &probes) {
    const uint32_t lane = lane_id();
    uint32_t k0 = 0, best = 0xFFFFFFFFu;
    for (uint32_t k = 0; k < nkeys; k++)
        if (((mask >> k) & 1u) && S.t_size[k] < best) {
            best = S.t_size[k];
            k0 = k;
        }
    if (lane < nkeys) S.t_cur[lane] = 0;
    __syncwarp();
    const bool old0 = __ldg(&T->key_old[k0]) != 0;
    uint32_t cnt = 0;
    for (uint32_t base = 0; base < best; base += 32) {
        const uint32_t idx = base + lane;
        bool ok = idx < best;
        uint32_t w = 0;
        if (ok) {
            const uint32_t e = __ldg(P.g.pool + S.t_off[k0] + idx);
            w = e >> 1;
            ok = !(old0 && (e & 1u));
            if (w >= P.g.V) {
                record_bad(P, CSM_BAD_ENTRY, e, S.t_off[k0] + idx, 700 + E);
                ok = false;
            }
        }
        for (uint32_t z = 0; ok && z < E; z++) ok = S.f[z] != w;
        const uint32_t vmask = __ballot_sync(0xffffffffu, idx < best);
        const uint32_t target = __shfl_sync(0xffffffffu, w, 31 - __clz(vmask));
        const uint32_t key_hi = (target + 1) << 1;
        for (uint32_t k = 0; k < nkeys; k++) {
            if (k == k0 || !((mask >> k) & 1u)) continue;
            if (!__any_sync(0xffffffffu, ok)) break;
            const uint32_t *L = P.g.pool + S.t_off[k];
            const uint32_t size = S.t_size[k], c0 = S.t_cur[k];
            const uint32_t win = c0 + lane < size ? __ldg(L + c0 + lane) : 0xFFFFFFFFu;
            const uint32_t below = __ballot_sync(0xffffffffu, win < key_hi);
            uint32_t e = 0xFFFFFFFFu, hi;
            if (below != 0xffffffffu) {
                hi = c0 + __popc(below);
                const uint32_t pos = shfl_lower_bound(win, w << 1);
                const uint32_t got = __shfl_sync(0xffffffffu, win, pos);
                if ((got >> 1) == w && got != 0xFFFFFFFFu) e = got;
            } else {
                hi = warp_lower_bound(L, c0 + 32, size, key_hi, lane);
                if (ok) e = find_entry(L + c0, hi - c0, w);
            }
            if (ok) {
                probes++;
                ok = e != 0xFFFFFFFFu && !(__ldg(&T->key_old[k]) && (e & 1u));
            }
            __syncwarp();
            if (lane == 0) S.t_cur[k] = hi;
            __syncwarp();
        }
        cnt += __popc(__ballot_sync(0xffffffffu, ok));
    }
    return cnt;
}

// Number of injective assignments of the tail vertices for the full prefix f[0..E-1].
__device__ unsigned long long tail_count(WarpState &S, const EnumParams &P, const DevPlan *pl,
                                         uint32_t &probes) {
    const uint32_t lane = lane_id();
    const DevTail *T = &pl->tail;
    const uint32_t nkeys = __ldg(&T->nkeys);
    const uint32_t nmasks = __ldg(&T->nmasks);
    const uint32_t E = pl->tail_start;
    // Lists whose size is used alone need their batch entries and the prefix vertices they
    // hold; intersections check both entry by entry.
    uint32_t single = 0;
    for (uint32_t mi = 0; mi < nmasks; mi++) {
        const uint32_t m = __ldg(&T->mask[mi]);
        if (__popc(m) == 1) single |= m;
    }
    if (lane < nkeys) {
        const uint32_t rel = __ldg(&T->key_rel[lane]);
        const uint32_t x = S.f[__ldg(&T->key_parent[lane])];
        const uint2 ms = list_of(P, rel, x, 300 + E);
        S.t_off[lane] = ms.x;
        S.t_size[lane] = ms.y;
        // Flagged entries of this list = batch edges of (rel, x) in this phase.
        S.t_flag[lane] = (__ldg(&T->key_old[lane]) && ((single >> lane) & 1u)) ? flagged_in_list(P, rel, x) : 0u;
        S.t_excl[lane] = 0;
    }
    __syncwarp();
    // Prefix vertices that sit in a list sized alone are not available to its vertex.
    uint32_t nprobe = 0;
    for (uint32_t pi = lane; pi < nkeys * E; pi += 32) {
        const uint32_t k = pi / E;
        if (!((single >> k) & 1u)) continue;
        if (!((__ldg(&T->key_excl[k]) >> (pi % E)) & 1u)) continue;  // other labels are never in the list
        const uint32_t z = S.f[pi % E];
        const uint32_t e = find_entry(P.g.pool + S.t_off[k], S.t_size[k], z);
        nprobe++;
        if (e != 0xFFFFFFFFu && !(__ldg(&T->key_old[k]) && (e & 1u))) atomicAdd(&S.t_excl[k], 1u);
    }
    probes += nprobe;
    __syncwarp();
    for (uint32_t mi = 0; mi < nmasks; mi++) {
        const uint32_t mask = __ldg(&T->mask[mi]);
        unsigned long long size;
        if (__popc(mask) == 1) {
            const uint32_t k = __ffs(mask) - 1;
            size = (unsigned long long)S.t_size[k] - S.t_flag[k] - S.t_excl[k];
        } else {
            size = tail_intersection(S, P, T, nkeys, mask, E, probes);
        }
        if (lane == 0) S.msize[mi] = size;
    }
    __syncwarp();
    unsigned long long total = 0;
    if (lane == 0) {
        total = 1;
        const DevTailTerm *terms = P.terms + pl->term_begin;
        const uint32_t nclasses = __ldg(&T->nclasses);
        for (uint32_t c = 0; c < nclasses; c++) {
            unsigned long long s = 0;
            const uint32_t tb = __ldg(&T->class_term_begin[c]), te = __ldg(&T->class_term_begin[c + 1]);
            for (uint32_t t = tb; t < te; t++) {
                unsigned long long prod = (unsigned long long)__ldg(&terms[t].coef);
                const uint32_t nf = __ldg(&terms[t].nf);
                for (uint32_t j = 0; j < nf; j++) prod *= S.msize[__ldg(&terms[t].f[j])];
                s += prod;
            }
            total *= s;
        }
    }
    __syncwarp();
    return total;
}

__device__ __forceinline__ unsigned long long slot_stamp(uint32_t epoch, uint32_t pos) {
    return ((unsigned long long)epoch << 32) | pos;
}

__device__ __forceinline__ unsigned long long device_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Checks the work item copied into S: plan, depth, candidate range and prefix vertex ids.  A
// failing item is recorded (`where`, `tag`) and must be skipped.  Warp-uniform.
__device__ bool item_ok(const WarpState &S, const EnumParams &P, uint32_t where, uint32_t tag) {
    const uint32_t lane = lane_id();
    const uint32_t plan = S.item_plan, depth = S.item_depth;
    bool ok = plan < P.nplans;
    if (ok) {
        if (depth == 0) ok = S.item_lo < S.item_hi && S.item_hi <= P.m;
        else ok = depth >= 2 && depth < P.plans[plan].n && S.item_lo <= S.item_hi;
    }
    const bool fok = !ok || lane >= depth || S.f[lane] < P.g.V;
    ok = __all_sync(0xffffffffu, ok && fok);
    if (!ok && lane == 0) record_bad(P, where, plan, depth, tag);
    __syncwarp();
    return ok;
}

// Reserves `cnt` (1..32) consecutive ring positions; returns the first, or 0xFFFFFFFF when the
// ring has no room (a full ring only costs balance: the donor keeps its work).  A position p of
// a later lap is free once the consumer of p - qcap has released its slot with stamp (epoch, p);
// first-lap positions are free as soon as nobody has reserved them.
__device__ uint32_t reserve_slots(const EnumParams &P, uint32_t cnt) {
    const uint32_t lane = lane_id();
    const uint32_t ep = P.ctrl->epoch;
    for (int tries = 0; tries < 16; tries++) {
        uint32_t pos = 0;
        if (lane == 0) pos = *(volatile unsigned int *)&P.ctrl->q_head;
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (pos > CSM_QUEUE_POS_LIMIT - cnt) break;
        const uint32_t p = pos + lane;
        bool free_slot = true;
        if (lane < cnt && p > P.qmask)
            free_slot = *(volatile unsigned long long *)(P.seq + (p & P.qmask)) == slot_stamp(ep, p);
        if (!__all_sync(0xffffffffu, free_slot)) break;
        uint32_t won = 0;
        if (lane == 0) won = atomicCAS(&P.ctrl->q_head, pos, pos + cnt) == pos;
        if (__shfl_sync(0xffffffffu, won, 0)) return pos;
    }
    if (lane == 0) atomicAdd(&P.ctrl->queue_full, 1ull);
    return 0xFFFFFFFFu;
}

// Writes the item of ring position `pos` and publishes it with stamp (epoch, pos + 1).
__device__ void publish_item(const EnumParams &P, uint32_t pos, uint32_t plan, uint32_t depth, uint32_t lo,
                             uint32_t hi, const uint32_t *prefix, uint32_t nprefix, bool extra, uint32_t extra_v,
                             uint32_t extra_pos) {
    const uint32_t lane = lane_id();
    WorkItem *it = P.queue + (pos & P.qmask);
    if (lane == 0) {
        it->plan = plan;
        it->depth = depth;
        it->lo = lo;
        it->hi = hi;
    }
    if (lane < nprefix) it->f[lane] = prefix[lane];
    if (extra && lane == 0) it->f[extra_pos] = extra_v;
    __threadfence();
    __syncwarp();
    if (lane == 0) atomicExch(P.seq + (pos & P.qmask), slot_stamp(P.ctrl->epoch, pos + 1));
    __syncwarp();
}

// Splits pending work of the current item into the queue.  Returns true if it donated.
__device__ bool try_donate(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t L0, uint32_t d) {
    const uint32_t lane = lane_id();
    const uint32_t E = pl->tail_start;
    // A shared last level is counted once per prefix at depth n - 3: the two deepest levels of
    // a prefix stay with the warp that holds it (so neither is counted twice).
    const uint32_t top = pl->shared_last ? pl->n - 3u : d;
    // Above a pendant counting level, buffered candidates are settled from the table, never
    // entered: they are not handed out as items of the counting level either.
    const uint32_t sib_end = pl->memo_slot != CSM_NO_MEMO ? E - 1u : E;
    for (uint32_t l = L0; l <= d && l <= top; l++) {
        const uint32_t lo = S.lo[l], hi = S.hi[l];
        const uint32_t minr = (l == 1) ? 64u : P.steal_min;
        if (hi > lo && hi - lo >= minr) {
            uint32_t mid = lo + ((hi - lo) >> 1);
            if (l == 1) mid = (mid + 31u) & ~31u;
            if (mid >= hi) continue;
            const uint32_t slot = reserve_slots(P, 1);
            if (slot == 0xFFFFFFFFu) return false;
            publish_item(P, slot, S.item_plan, l == 1 ? 0u : l, mid, hi, S.f, l == 1 ? 0u : l, false, 0, 0);
            if (lane == 0) {
                S.hi[l] = mid;
                atomicAdd(&P.ctrl->donations, 1ull);
            }
            __syncwarp();
            return true;
        }
        const uint32_t nb = S.nbuf[l], ps = S.pos[l];
        if (l < d && l + 1 < sib_end && nb > ps) {
            const uint32_t cnt = nb - ps;
            const uint32_t slot = reserve_slots(P, cnt);
            if (slot == 0xFFFFFFFFu) return false;
            for (uint32_t j = 0; j < cnt; j++) {
                const uint32_t c = S.buf[l][ps + j];
                if (l == 1) {
                    const unsigned long long key = __ldg(P.keys + c);
                    uint32_t pre[2] = {P.kl.src(key), P.kl.dst(key)};
                    publish_item(P, slot + j, S.item_plan, 2, 0, 0xFFFFFFFFu, pre, 2, false, 0, 0);
                } else {
                    publish_item(P, slot + j, S.item_plan, l + 1, 0, 0xFFFFFFFFu, S.f, l, true, c, l);
                }
            }
            if (lane == 0) {
                S.nbuf[l] = (uint8_t)ps;
                atomicAdd(&P.ctrl->donations, (unsigned long long)cnt);
            }
            __syncwarp();
            return true;
        }
    }
    return false;
}

// Claims the oldest published item into S; returns 1 on success, 0 when none is ready.  The
// position at the ring's tail is taken only once its item is published, so a claim never waits;
// after copying the item the slot is released for the position one lap later.
__device__ int claim_item(WarpState &S, const EnumParams &P) {
    const uint32_t lane = lane_id();
    const uint32_t ep = P.ctrl->epoch;
    uint32_t pos = 0xFFFFFFFFu;
    if (lane == 0) {
        volatile unsigned int *qt = &P.ctrl->q_tail;
        for (int tries = 0; tries < 64; tries++) {
            const uint32_t t = *qt;
            const unsigned long long sq = *(volatile unsigned long long *)(P.seq + (t & P.qmask));
            if (sq != slot_stamp(ep, t + 1)) {
                if (*qt == t) break;  // the tail's item is not published yet: nothing ready
                continue;             // another warp took it; look at the new tail
            }
            if (atomicCAS(&P.ctrl->q_tail, t, t + 1) == t) {
                pos = t;
                break;
            }
        }
        __threadfence();
    }
    pos = __shfl_sync(0xffffffffu, pos, 0);
    if (pos == 0xFFFFFFFFu) return 0;
    volatile const WorkItem *it = P.queue + (pos & P.qmask);
    if (lane == 0) {
        S.item_plan = it->plan;
        S.item_depth = it->depth;
        S.item_lo = it->lo;
        S.item_hi = it->hi;
    }
    if (lane < CSM_MAXQV) S.f[lane] = it->f[lane];
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        atomicExch(P.seq + (pos & P.qmask), slot_stamp(ep, pos + P.qmask + 1));
    }
    __syncwarp();
    return item_ok(S, P, CSM_BAD_ITEM, pos) ? 1 : 0;
}

// Withdraws one outstanding work request (an idle warp that leaves without work).
__device__ void withdraw_request(const EnumParams &P) {
    unsigned int h = *(volatile unsigned int *)&P.ctrl->hungry;
    for (int tries = 0; tries < 64 && h > 0; tries++) {
        const unsigned int prev = atomicCAS(&P.ctrl->hungry, h, h - 1);
        if (prev == h) return;
        h = prev;
    }
}

// Takes the next seed chunk or frontier item into S: 1 = taken, 0 = none left, -1 = a frontier
// item that failed its check (skipped).
__device__ int take_ticket(WarpState &S, const EnumParams &P) {
    const uint32_t lane = lane_id();
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&P.ctrl->ticket, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    const unsigned long long nt = *(volatile unsigned long long *)&P.ctrl->nticket;
    if (t >= nt) return 0;
    if (P.frontier != nullptr) {
        const WorkItem *it = P.frontier + t;
        if (lane == 0) {
            S.item_plan = it->plan;
            S.item_depth = it->depth;
            S.item_lo = it->lo;
            S.item_hi = it->hi;
        }
        if (lane < CSM_MAXQV) S.f[lane] = it->f[lane];
        __syncwarp();
        if (!item_ok(S, P, CSM_BAD_FRONTIER, (uint32_t)t)) return -1;
    } else {
        // Seed chunk t: plan p with ticket_prefix[p] <= t < ticket_prefix[p+1].
        uint32_t lo = 0, hi = P.nplans;
        while (lo + 1 < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (__ldg(P.ticket_prefix + mid) <= t) lo = mid;
            else hi = mid;
        }
        const uint32_t p = lo;
        const uint32_t chunk = (uint32_t)(t - __ldg(P.ticket_prefix + p));
        const uint32_t s0 = __ldg(P.seed_lo + p) + chunk * 32u;
        const uint32_t s_end = __ldg(P.seed_lo + P.nplans + p);
        if (lane == 0) {
            S.item_plan = p;
            S.item_depth = 0;
            S.item_lo = s0;
            S.item_hi = s0 + 32u < s_end ? s0 + 32u : s_end;
        }
    }
    __syncwarp();
    return 1;
}

__device__ void write_row(const EnumParams &P, const DevPlan *pl, const WarpState &S, uint32_t d, uint32_t w,
                          unsigned long long r) {
    uint32_t *row = P.rows + r * CSM_ROW_WORDS;
    row[0] = pl->query;
    for (uint32_t k = 0; k < d; k++) row[1 + pl->order[k]] = S.f[k];
    row[1 + pl->order[d]] = w;
}

// Last counting level with packed siblings.  The buffered candidates s_0..s_{k-1} of level
// d = n - 2 each open a last level whose candidate lists are usually short, so instead of one
// pass per sibling the warp scans all their pivot lists at once, one (sibling, position) pair
// per lane.  A lane finds its sibling by a shuffle search over the inclusive prefix of list
// lengths and checks its candidate like the per-sibling scan (flag rule, injectivity, NLF
// bitmap, membership in the other backward lists by binary search).  Returns false (nothing
// counted) when the lists are long enough for the per-sibling scan to fill the warp.
__device__ bool count_last_packed(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t d,
                                  unsigned long long &cnt, uint32_t &scans, uint32_t &probes) {
    const uint32_t lane = lane_id();
    const uint32_t L = d + 1;
    const DevLevel *lv = &pl->lv[L];
    const uint32_t nbn = __ldg(&lv->nbn);
    const uint32_t oldm = __ldg(&lv->old_mask);
    const uint32_t nlf_id = __ldg(&lv->nlf_bitmap);
    const uint32_t *nlf = nlf_id == CSM_NO_BITMAP ? nullptr : bitmap(P, nlf_id);
    const uint32_t exm = __ldg(&lv->excl_mask) & ((1u << d) - 1u);  // depth d is the sibling itself
    const uint32_t ps = S.pos[d], k = S.nbuf[d] - ps;
    // Shared lists: backward neighbours matched before depth d (same for every sibling).
    // sib_b = the backward neighbour at depth d (at most one), whose list is the sibling's own.
    const uint32_t bb = __ldg(&lv->bn_base);
    uint32_t sib_b = 0xFFu, sh_min = 0xFFFFFFFFu, sh_piv = 0;
    for (uint32_t b = 0; b < nbn; b++) {
        const uint32_t dep = __ldg(&lv->bn_depth[b]);
        if (dep == d) {
            sib_b = b;
            continue;
        }
        const uint2 ms = list_of(P, __ldg(&lv->bn_rel[b]), S.f[dep], 400 + L);
        if (lane == 0) {
            S.poff[bb + b] = ms.x;  // level L's own slots: it is counted, never entered
            S.psz[bb + b] = ms.y;
        }
        if (ms.y < sh_min) {
            sh_min = ms.y;
            sh_piv = b;
        }
    }
    __syncwarp();
    // Per sibling (lane j < k): its own list, its pivot and the pivot's list.
    uint32_t sv = 0, s_off = 0, s_sz = 0, pv = sh_piv, p_off = 0, p_len = 0;
    if (lane < k) {
        sv = S.buf[d][ps + lane];
        if (sib_b != 0xFFu) {
            const uint2 ms = list_of(P, __ldg(&lv->bn_rel[sib_b]), sv, 500 + L);
            s_off = ms.x;
            s_sz = ms.y;
        }
        // The smallest list is the pivot, the lowest backward-neighbour index on ties (the
        // choice enter_level makes), so the work counters do not depend on packing.
        if (sib_b != 0xFFu && (s_sz < sh_min || (s_sz == sh_min && sib_b < sh_piv))) {
            pv = sib_b;
            p_off = s_off;
            p_len = s_sz;
        } else {
            p_off = S.poff[bb + sh_piv];
            p_len = sh_min;
        }
    }
    // Inclusive prefix of pivot lengths.
    uint32_t incl = p_len;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total > 4u * k) return false;  // longer lists: the per-sibling scan fills the warp better
    for (uint32_t g0 = 0; g0 < total; g0 += 32) {
        const uint32_t g = g0 + lane;
        // Sibling of position g: the first lane whose inclusive prefix exceeds g.
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0; step >>= 1)
            if (__shfl_sync(0xffffffffu, incl, j + step - 1) <= g) j += step;
        const uint32_t jc = j < 31 ? j : 31;
        const uint32_t excl_j = __shfl_sync(0xffffffffu, incl, jc) - __shfl_sync(0xffffffffu, p_len, jc);
        const uint32_t c_sv = __shfl_sync(0xffffffffu, sv, jc);
        const uint32_t c_soff = __shfl_sync(0xffffffffu, s_off, jc);
        const uint32_t c_ssz = __shfl_sync(0xffffffffu, s_sz, jc);
        const uint32_t c_pv = __shfl_sync(0xffffffffu, pv, jc);
        const uint32_t c_poff = __shfl_sync(0xffffffffu, p_off, jc);
        bool ok = g < total;
        uint32_t w = 0;
        if (ok) {
            const uint32_t e = __ldg(P.g.pool + c_poff + (g - excl_j));
            w = e >> 1;
            scans++;
            ok = !(((oldm >> c_pv) & 1u) && (e & 1u)) && w != c_sv;
            if (w >= P.g.V) {
                record_bad(P, CSM_BAD_ENTRY, e, c_poff + (g - excl_j), 600 + L);
                ok = false;
            }
        }
        for (uint32_t em = exm; ok && em; em &= em - 1) ok = S.f[__ffs(em) - 1] != w;
        const uint32_t nlf_word = !ok ? 0u : (nlf ? __ldg(nlf + (w >> 5)) : 0xFFFFFFFFu);
        for (uint32_t b = 0; ok && b < nbn; b++) {
            if (b == c_pv) continue;
            const uint32_t *list = b == sib_b ? P.g.pool + c_soff : P.g.pool + S.poff[bb + b];
            const uint32_t sz = b == sib_b ? c_ssz : S.psz[bb + b];
            const uint32_t e = find_entry(list, sz, w);
            probes++;
            ok = e != 0xFFFFFFFFu && !(((oldm >> b) & 1u) && (e & 1u));
        }
        if (ok) ok = (nlf_word >> (w & 31)) & 1u;
        cnt += __popc(__ballot_sync(0xffffffffu, ok));
    }
    __syncwarp();
    if (lane == 0) S.pos[d] = S.nbuf[d];
    __syncwarp();
    return true;
}

// Last level of a counting plan without a tail: the matches are the pivot-list candidates that
// pass the flag rule, injectivity and membership in the one other backward list, i.e. a
// filtered count of a sorted-list intersection (the shape of the last level of every dense plan
// measured: two backward neighbours).  The other list's offset, size, cursor and flag rule stay
// in registers for the whole scan instead of being re-read from the warp's shared state for
// every 32 candidates.  Every 8 chunks the warp answers work requests (donating the upper half
// of the remaining range) and checks the time limit.  Returns the count; the level is left
// exhausted (S.lo[d] >= S.hi[d]).
constexpr uint32_t kLastLists = 1;
constexpr uint32_t kWindows = 3;

__device__ unsigned long long count_last_level(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t L0,
                                               uint32_t d, uint32_t &scans, uint32_t &probes, unsigned int &err,
                                               unsigned long long deadline) {
    const uint32_t lane = lane_id();
    const uint32_t nbn = S.nbn[d], piv = S.piv[d], bb = S.bnb[d];
    const uint32_t oldm = S.oldm[d], exm = S.exm[d], nlf_id = S.nlf[d];
    const bool piv_old = (oldm >> piv) & 1u;
    const uint32_t *nlf = nlf_id == CSM_NO_BITMAP ? nullptr : bitmap(P, nlf_id);
    const uint32_t *base = P.g.pool + S.base[d];
    uint32_t l_off[kLastLists], l_size[kLastLists], l_cur[kLastLists];
    uint32_t l_old = 0;  // bit j: list j's batch entries do not count
    uint32_t nl = 0;
#pragma unroll
    for (uint32_t j = 0; j < kLastLists; j++) l_off[j] = l_size[j] = l_cur[j] = 0;
    for (uint32_t k = 0; k < nbn; k++) {
        if (k == piv) continue;
#pragma unroll
        for (uint32_t j = 0; j < kLastLists; j++)
            if (j == nl) {
                l_off[j] = S.poff[bb + k];
                l_size[j] = S.psz[bb + k];
                l_old |= ((oldm >> k) & 1u) << j;
            }
        nl++;
    }
    uint32_t lo = S.lo[d], hi = S.hi[d];
    unsigned long long cnt = 0;
    for (uint32_t chunk = 1; lo < hi; lo += 32, chunk++) {
        const uint32_t idx = lo + lane;
        const bool in = idx < hi;
        bool ok = in;
        uint32_t cand = 0;
        if (ok) {
            const uint32_t e = __ldg(base + idx);
            cand = e >> 1;
            scans++;
            ok = !(piv_old && (e & 1u));
            if (cand >= P.g.V) {
                record_bad(P, CSM_BAD_ENTRY, e, S.base[d] + idx, d);
                ok = false;
            }
        }
        for (uint32_t em = exm; ok && em; em &= em - 1) ok = S.f[__ffs(em) - 1] != cand;
        const uint32_t nlf_word = !ok ? 0u : (nlf ? __ldg(nlf + (cand >> 5)) : 0xFFFFFFFFu);
        const uint32_t vmask = __ballot_sync(0xffffffffu, in);
        const uint32_t target = __shfl_sync(0xffffffffu, cand, 31 - __clz(vmask));
        const uint32_t key_hi = (target + 1) << 1;
        uint32_t win[kLastLists];
#pragma unroll
        for (uint32_t j = 0; j < kLastLists; j++)
            win[j] = (j < nl && l_cur[j] + lane < l_size[j]) ? __ldg(P.g.pool + l_off[j] + l_cur[j] + lane) : 0xFFFFFFFFu;
#pragma unroll
        for (uint32_t j = 0; j < kLastLists; j++) {
            if (j >= nl) break;
            uint32_t e = 0xFFFFFFFFu, nhi = 0;
            // The chunk's candidates span ~40-55 entries of the other list on the measured
            // queries: walk up to kWindows consecutive 32-entry windows (one coalesced load each)
            // before bracketing the rest of the list with the warp search.
            const uint32_t *L = P.g.pool + l_off[j];
            uint32_t c0 = l_cur[j], w = win[j];
            bool done = false;
#pragma unroll 1
            for (uint32_t k = 0; k < kWindows; k++) {
                const uint32_t below = __ballot_sync(0xffffffffu, w < key_hi);
                const uint32_t pos = shfl_lower_bound(w, cand << 1);
                const uint32_t got = __shfl_sync(0xffffffffu, w, pos);
                if ((got >> 1) == cand && got != 0xFFFFFFFFu) e = got;
                if (below != 0xffffffffu) {
                    nhi = c0 + __popc(below);
                    done = true;
                    break;
                }
                c0 += 32;
                w = c0 + lane < l_size[j] ? __ldg(L + c0 + lane) : 0xFFFFFFFFu;
            }
            if (!done) {
                nhi = warp_lower_bound(L, c0, l_size[j], key_hi, lane);
                if (ok && e == 0xFFFFFFFFu) e = find_entry(L + c0, nhi - c0, cand);
            }
            if (ok) {
                probes++;
                ok = e != 0xFFFFFFFFu && !(((l_old >> j) & 1u) && (e & 1u));
            }
            l_cur[j] = nhi;
        }
        if (ok) ok = (nlf_word >> (cand & 31)) & 1u;
        cnt += __popc(__ballot_sync(0xffffffffu, ok));
        if ((chunk & 7u) == 0 && lo + 32 < hi) {
            if (deadline) {
                unsigned int late = 0;
                if (lane == 0) late = device_ns() > deadline;
                if (__shfl_sync(0xffffffffu, late, 0)) {
                    err |= CSM_ERRBIT_TIMEOUT;
                    break;
                }
            }
            if (P.donate) {
                unsigned int granted = 0;
                if (lane == 0) {
                    const unsigned int h = *(volatile unsigned int *)&P.ctrl->hungry;
                    granted = h > 0 && atomicCAS(&P.ctrl->hungry, h, h - 1) == h;
                }
                if (__shfl_sync(0xffffffffu, granted, 0)) {
                    // The remaining range [lo + 32, hi) is this level's pending work.
                    if (lane == 0) {
                        S.lo[d] = lo + 32;
                        S.hi[d] = hi;
                    }
                    __syncwarp();
                    if (!try_donate(S, P, pl, L0, d) && lane == 0) atomicAdd(&P.ctrl->hungry, 1u);
                    hi = S.hi[d];
                    __syncwarp();
                }
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        S.lo[d] = hi;
        S.hi[d] = hi;
    }
    __syncwarp();
    return cnt;
}

// Shared last level (DevPlan.shared_last), level d = n - 2 with candidates buffered: the count
// of the last level for the prefix f[0..n-3] was taken once (S.sl_count, with f[n-2] left out of
// its exclusions), so each buffered candidate v contributes that count, minus one when v is
// itself a candidate of the last level — in every backward list of level n - 1 under the flag
// rule and in its NLF bitmap.  v differs from every prefix vertex of its own label already, so
// nothing else changes.  Consumes the buffer.
__device__ unsigned long long count_shared_last(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t d,
                                                uint32_t &probes) {
    const uint32_t lane = lane_id();
    const uint32_t L = d + 1;
    const uint32_t ps = S.pos[d], k = S.nbuf[d] - ps;
    unsigned long long total = (unsigned long long)k * S.sl_count;
    if ((__ldg(&pl->lv[L].excl_mask) >> d) & 1u) {
        bool in = lane < k;
        if (in) {
            const uint32_t v = S.buf[d][ps + lane];
            const uint32_t nbn = S.nbn[L], bb = S.bnb[L], oldm = S.oldm[L], nlf_id = S.nlf[L];
            for (uint32_t b = 0; in && b < nbn; b++) {
                const uint32_t e = find_entry(P.g.pool + S.poff[bb + b], S.psz[bb + b], v);
                probes++;
                in = e != 0xFFFFFFFFu && !(((oldm >> b) & 1u) && (e & 1u));
            }
            if (in && nlf_id != CSM_NO_BITMAP) in = test_bit(bitmap(P, nlf_id), v);
        }
        total -= __popc(__ballot_sync(0xffffffffu, in));
    }
    __syncwarp();
    if (lane == 0) S.pos[d] = S.nbuf[d];
    __syncwarp();
    return total;
}

// Pendant counting level c = d + 1 (DevPlan.memo_slot): every buffered candidate of level d
// contributes the table entry of the data vertex at memo_depth (the candidate itself when that
// depth is d).  Consumes the buffer.
__device__ unsigned long long settle_pendant(WarpState &S, const EnumParams &P, const DevPlan *pl, uint32_t d,
                                             uint32_t &tails) {
    const uint32_t lane = lane_id();
    const uint32_t ps = S.pos[d], k = S.nbuf[d] - ps;
    const uint32_t md = pl->memo_depth;
    const unsigned long long *table = P.memo + (size_t)pl->memo_slot * P.g.V;
    unsigned long long v = 0;
    if (lane < k) {
        const uint32_t x = md == d ? S.buf[d][ps + lane] : S.f[md];
        v = __ldg(table + x);
    }
    tails += k;  // warp-uniform, like every other use of the tail counter
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncwarp();
    if (lane == 0) S.pos[d] = S.nbuf[d];
    __syncwarp();
    return v;
}

// Runs one work item to completion (or until the device clock passes `deadline`, when that is
// nonzero: the rest of the item is then dropped and CSM_ERRBIT_TIMEOUT set).  Returns the number
// of matches counted.
template <bool LASTLOOP, int MODE>
__device__ unsigned long long run_item(WarpState &S, const EnumParams &P, uint32_t &scans,
                                       uint32_t &probes, uint32_t &tails, uint32_t &shared, unsigned int &err,
                                       unsigned long long deadline) {
    const uint32_t lane = lane_id();
    const DevPlan *pl = P.plans + S.item_plan;
    const uint32_t n = pl->n;
    const uint32_t E = pl->tail_start;
    const uint32_t L0 = S.item_depth == 0 ? 1u : S.item_depth;
    unsigned long long cnt = 0;

    if (MODE == CSM_ENUM_MODE_EXPAND && L0 >= pl->expand_stop) {
        // Nothing left to expand before the counting level: pass the item through.
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(&P.ctrl->out_rows, 1ull);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r < P.expand_cap) {
            WorkItem *o = P.expand_out + r;
            if (lane == 0) {
                o->plan = S.item_plan;
                o->depth = S.item_depth;
                o->lo = S.item_lo;
                o->hi = S.item_hi;
            }
            if (lane < CSM_MAXQV) o->f[lane] = S.f[lane];
        } else if (lane == 0) {
            err |= CSM_ERRBIT_OUTPUT;
        }
        __syncwarp();
        return 0;
    }

    if (L0 == 1) {
        if (lane == 0) {
            S.lo[1] = S.item_lo;
            S.hi[1] = S.item_hi;
            S.nbuf[1] = 0;
            S.pos[1] = 0;
        }
        __syncwarp();
    } else {
        enter_level(S, P, pl, L0, S.item_lo, S.item_hi);
    }
    uint32_t d = L0;
    uint32_t iter = 0;
    unsigned long long sl_before = 0;
    if (lane == 0) S.sl_state = 0;
    const uint32_t *nlf0 = bitmap(P, pl->nlf0);
    const uint32_t *nlf1 = bitmap(P, pl->nlf1);

    while (true) {
        ++iter;
        if (deadline && (iter & 63u) == 0) {
            unsigned int late = 0;
            if (lane == 0) late = device_ns() > deadline;
            if (__shfl_sync(0xffffffffu, late, 0)) {
                err |= CSM_ERRBIT_TIMEOUT;
                break;
            }
        }
        if (P.donate && (iter & 7u) == 0) {
            // Each idle warp posts one request; a busy warp that takes a request splits off
            // one piece of its pending work (and hands the request back if it has none).
            unsigned int granted = 0;
            if (lane == 0) {
                const unsigned int h = *(volatile unsigned int *)&P.ctrl->hungry;
                granted = h > 0 && atomicCAS(&P.ctrl->hungry, h, h - 1) == h;
            }
            granted = __shfl_sync(0xffffffffu, granted, 0);
            if (granted && !try_donate(S, P, pl, L0, d) && lane == 0) atomicAdd(&P.ctrl->hungry, 1u);
        }
        if (S.pos[d] < S.nbuf[d]) {
            if (MODE == CSM_ENUM_MODE_COUNT && d + 2 == E && P.memo != nullptr && pl->memo_slot < CSM_MEMO_PENDING) {
                // Pendant counting level below: each buffered candidate's count is a table entry.
                cnt += settle_pendant(S, P, pl, d, tails);
                continue;
            }
            if (MODE == CSM_ENUM_MODE_COUNT && d + 2 == n && pl->shared_last) {
                // The last level does not depend on these candidates: count it once for the
                // prefix (first time here), then settle every buffered candidate at once.
                if (S.sl_state == 2) {
                    cnt += count_shared_last(S, P, pl, d, probes);
                    continue;
                }
                sl_before = cnt;
                shared++;
                d++;
                enter_level(S, P, pl, d, 0, 0xFFFFFFFFu);
                if (lane == 0) {
                    S.sl_state = 1;
                    S.exm[d] &= (uint16_t)~(1u << (d - 1));  // f[n-2] is settled per candidate
                }
                __syncwarp();
                continue;
            }
            // Siblings whose subtree is only the last level: count them together.  Tried once per
            // buffer: when the lists are too long for it, they stay so for the later siblings.
            if (d + 2 == n && E == n && d >= 2 && MODE == CSM_ENUM_MODE_COUNT && S.pos[d] == 0 &&
                count_last_packed(S, P, pl, d, cnt, scans, probes))
                continue;
            // Descend into the next buffered candidate.
            const uint32_t c = S.buf[d][S.pos[d]];
            __syncwarp();
            if (lane == 0) {
                S.pos[d]++;
                if (d == 1) {
                    const unsigned long long key = __ldg(P.keys + c);
                    S.f[0] = P.kl.src(key);
                    S.f[1] = P.kl.dst(key);
                } else {
                    S.f[d] = c;
                }
            }
            __syncwarp();
            if (d + 1 == E) {
                cnt += tail_count(S, P, pl, probes);
                tails++;
            } else {
                d++;
                if (lane == 0 && d + 2 == n) S.sl_state = 0;  // a new prefix f[0..n-3]
                enter_level(S, P, pl, d, 0, 0xFFFFFFFFu);
            }
            continue;
        }
        if (S.lo[d] >= S.hi[d]) {
            if (MODE == CSM_ENUM_MODE_COUNT && d + 1 == n && S.sl_state == 1) {
                // The shared last level is counted: keep its count for the candidates above.
                if (lane == 0) {
                    S.sl_count = cnt - sl_before;
                    S.sl_state = 2;
                }
                cnt = sl_before;
                __syncwarp();
            }
            if (d == L0) break;
            d--;
            continue;
        }
        if (LASTLOOP && d + 1 == n && E == n && d >= 2 && MODE == CSM_ENUM_MODE_COUNT && S.nbn[d] <= kLastLists + 1) {
            cnt += count_last_level(S, P, pl, L0, d, scans, probes, err, deadline);
            if (err & CSM_ERRBIT_TIMEOUT) break;
            continue;
        }
        // Scan the next 32 candidates of level d.
        const uint32_t idx = S.lo[d] + lane;
        bool ok = idx < S.hi[d];
        uint32_t cand = 0;
        if (d == 1) {
            if (ok) {
                const unsigned long long key = __ldg(P.keys + idx);
                const uint32_t x = P.kl.src(key), y = P.kl.dst(key);
                ok = __ldg(P.eff + idx) == P.phase && x != y && test_bit(nlf0, x) && test_bit(nlf1, y);
                cand = idx;
            }
        } else {
            const uint32_t oldm = S.oldm[d];
            const uint32_t piv = S.piv[d];
            if (ok) {
                const uint32_t e = __ldg(P.g.pool + S.base[d] + idx);
                cand = e >> 1;
                scans++;
                ok = !(((oldm >> piv) & 1u) && (e & 1u));
                if (cand >= P.g.V) {
                    record_bad(P, CSM_BAD_ENTRY, e, S.base[d] + idx, d);
                    ok = false;
                }
            }
            for (uint32_t em = S.exm[d]; ok && em; em &= em - 1) ok = S.f[__ffs(em) - 1] != cand;
            // The NLF word is loaded now and tested after the probes, so its latency overlaps
            // theirs (probes are warp-wide and do not depend on it).
            const uint32_t nlf_id = S.nlf[d];
            const uint32_t nlf_word =
                !ok ? 0u : (nlf_id == CSM_NO_BITMAP ? 0xFFFFFFFFu : __ldg(bitmap(P, nlf_id) + (cand >> 5)));
            // Membership in the other backward lists.  The chunk's candidates ascend, so each
            // list keeps a cursor.  The 32 entries at the cursor are read first: when they
            // reach past the chunk's largest candidate, the window is in registers and
            // shuffles find each candidate (one dependent read).  Otherwise a 32-ary warp search
            // brackets the window and lanes search inside it.
            const uint32_t nbn = S.nbn[d];
            const uint32_t vmask = __ballot_sync(0xffffffffu, idx < S.hi[d]);
            const uint32_t target = __shfl_sync(0xffffffffu, cand, 31 - __clz(vmask));
            const uint32_t key_hi = (target + 1) << 1;
            // The windows of up to four lists are read together (independent loads in flight
            // at once), then each list is resolved in turn.
            for (uint32_t k0 = 0; k0 < nbn; k0 += 4) {
                if (!__any_sync(0xffffffffu, ok)) break;
                uint32_t win[4];
#pragma unroll
                for (uint32_t j = 0; j < 4; j++) {
                    const uint32_t k = k0 + j;
                    win[j] = 0xFFFFFFFFu;
                    if (k < nbn && k != piv) {
                        const uint32_t slot = S.bnb[d] + k;
                        const uint32_t c0 = S.cur[slot];
                        if (c0 + lane < S.psz[slot]) win[j] = __ldg(P.g.pool + S.poff[slot] + c0 + lane);
                    }
                }
#pragma unroll
                for (uint32_t j = 0; j < 4; j++) {
                    const uint32_t k = k0 + j;
                    if (k >= nbn || k == piv) continue;
                    if (!__any_sync(0xffffffffu, ok)) break;
                    const uint32_t slot = S.bnb[d] + k;
                    const uint32_t *L = P.g.pool + S.poff[slot];
                    const uint32_t c0 = S.cur[slot];
                    const uint32_t size = S.psz[slot];
                    const uint32_t below = __ballot_sync(0xffffffffu, win[j] < key_hi);
                    uint32_t e = 0xFFFFFFFFu, hi;
                    if (below != 0xffffffffu) {
                        // The window [c0, hi) fits in the 32 entries just read.
                        hi = c0 + __popc(below);
                        const uint32_t pos = shfl_lower_bound(win[j], cand << 1);
                        const uint32_t got = __shfl_sync(0xffffffffu, win[j], pos);
                        if ((got >> 1) == cand && got != 0xFFFFFFFFu) e = got;
                    } else {
                        hi = warp_lower_bound(L, c0 + 32, size, key_hi, lane);
                        if (ok) e = find_entry(L + c0, hi - c0, cand);
                    }
                    if (ok) {
                        probes++;
                        ok = e != 0xFFFFFFFFu && !(((oldm >> k) & 1u) && (e & 1u));
                    }
                    if (lane == 0) S.cur[slot] = hi;
                }
            }
            if (ok) ok = (nlf_word >> (cand & 31)) & 1u;
        }
        __syncwarp();
        if (lane == 0) S.lo[d] += 32u;
        const uint32_t mask = __ballot_sync(0xffffffffu, ok);
        const uint32_t rank = __popc(mask & ((1u << lane) - 1u));
        if (MODE == CSM_ENUM_MODE_EXPAND && d == L0) {
            // One BFS level: survivors become items of depth d + 1.
            const uint32_t c = __popc(mask);
            unsigned long long r = 0;
            if (lane == 0 && c) r = atomicAdd(&P.ctrl->out_rows, (unsigned long long)c);
            r = __shfl_sync(0xffffffffu, r, 0);
            if (c && r + c > P.expand_cap) {
                if (lane == 0) err |= CSM_ERRBIT_OUTPUT;
            } else if (ok) {
                WorkItem *o = P.expand_out + r + rank;
                o->plan = S.item_plan;
                o->depth = d + 1;
                o->lo = 0;
                o->hi = 0xFFFFFFFFu;
                if (d == 1) {
                    const unsigned long long key = __ldg(P.keys + cand);
                    o->f[0] = P.kl.src(key);
                    o->f[1] = P.kl.dst(key);
                } else {
                    for (uint32_t k = 0; k < d; k++) o->f[k] = S.f[k];
                    o->f[d] = cand;
                }
            }
            __syncwarp();
        } else if (d + 1 == E && E < n && pl->tail.lane_par) {
            // Counting level before the tail: every surviving lane sizes its own tail.  Lists
            // shared by the chunk (parent matched above this level) are searched by the warp
            // with a cursor, as the probe lists are: the chunk's candidates ascend.
            uint32_t shared_hit = 0;
            if (d >= 2) {
                const DevTail *T = &pl->tail;
                const uint32_t nkeys = __ldg(&T->nkeys);
                const uint32_t vm = __ballot_sync(0xffffffffu, idx < S.hi[d]);
                const uint32_t tgt = __shfl_sync(0xffffffffu, cand, 31 - __clz(vm));
                const uint32_t key_hi = (tgt + 1) << 1;
                for (uint32_t k = 0; k < nkeys; k++) {
                    if (__ldg(&T->key_parent[k]) >= d) continue;
                    if (!((__ldg(&T->key_excl[k]) >> d) & 1u)) continue;  // candidates never in this list
                    if (!__any_sync(0xffffffffu, ok)) break;
                    const uint32_t *L = P.g.pool + S.ts_off[k];
                    const uint32_t size = S.ts_size[k];
                    const uint32_t c0 = S.ts_cur[k];
                    const uint32_t win = c0 + lane < size ? __ldg(L + c0 + lane) : 0xFFFFFFFFu;
                    const uint32_t below = __ballot_sync(0xffffffffu, win < key_hi);
                    uint32_t e = 0xFFFFFFFFu, hi;
                    if (below != 0xffffffffu) {
                        hi = c0 + __popc(below);
                        const uint32_t pos = shfl_lower_bound(win, cand << 1);
                        const uint32_t got = __shfl_sync(0xffffffffu, win, pos);
                        if ((got >> 1) == cand && got != 0xFFFFFFFFu) e = got;
                    } else {
                        hi = warp_lower_bound(L, c0 + 32, size, key_hi, lane);
                        if (ok) e = find_entry(L + c0, hi - c0, cand);
                    }
                    __syncwarp();
                    if (lane == 0) S.ts_cur[k] = hi;
                    if (ok) {
                        probes++;
                        const bool old_k = __ldg(&T->key_old[k]) != 0;
                        if (e != 0xFFFFFFFFu && !(old_k && (e & 1u))) shared_hit |= 1u << k;
                    }
                }
                __syncwarp();
            }
            unsigned long long t = 0;
            if (ok) {
                if (d == 1) {
                    const unsigned long long key = __ldg(P.keys + cand);
                    t = tail_count_lane(S.ts_base, S.f, P, pl, 1, P.kl.src(key), P.kl.dst(key), 0, probes);
                } else {
                    t = tail_count_lane(S.ts_base, S.f, P, pl, d, 0, cand, shared_hit, probes);
                }
            }
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            cnt += t;
            tails += __popc(mask);
        } else if (d + 1 == n) {
            if (MODE == CSM_ENUM_MODE_ROWS) {
                const uint32_t c = __popc(mask);
                unsigned long long r = 0;
                if (lane == 0 && c) r = atomicAdd(&P.ctrl->out_rows, (unsigned long long)c);
                r = __shfl_sync(0xffffffffu, r, 0);
                if (c && r + c > P.row_cap) {
                    if (lane == 0) err |= CSM_ERRBIT_OUTPUT;
                } else if (ok) {
                    if (d == 1) {
                        const unsigned long long key = __ldg(P.keys + cand);
                        uint32_t *row = P.rows + (r + rank) * CSM_ROW_WORDS;
                        row[0] = pl->query;
                        row[1 + pl->order[0]] = P.kl.src(key);
                        row[1 + pl->order[1]] = P.kl.dst(key);
                    } else {
                        write_row(P, pl, S, d, cand, r + rank);
                    }
                }
            }
            cnt += __popc(mask);
            __syncwarp();
        } else {
            if (ok) S.buf[d][rank] = cand;
            __syncwarp();
            if (lane == 0) {
                S.nbuf[d] = (uint8_t)__popc(mask);
                S.pos[d] = 0;
            }
            __syncwarp();
        }
    }
    return cnt;
}

// MINB resident blocks of 256 threads per SM: the register budget per thread follows from it.
// MODE: CSM_ENUM_MODE_* of the launch (each variant holds only its mode's code, which keeps the
// hot loop's instruction footprint small).
template <int MINB, bool LASTLOOP, int MODE>
__global__ void __launch_bounds__(256, MINB) k_enumerate(EnumParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    WarpState &S = reinterpret_cast<WarpState *>(smem)[threadIdx.x >> 5];
    const uint32_t lane = lane_id();
    if (P.abort_flag != nullptr && *(volatile const unsigned int *)P.abort_flag) return;
    // Per-lane work counters (statistics only), 32-bit to keep registers for the search; a
    // lane flushes them to the launch totals before they could wrap.
    uint32_t scans = 0, probes = 0, tails = 0, shared = 0;
    unsigned int err = 0;
    const unsigned long long deadline = P.time_limit_ns ? P.ctrl->t_start + P.time_limit_ns : 0ull;
    bool have_source = true;  // seed tickets / frontier not yet exhausted
    // A warp counts as active from its start: blocks that become resident late (the GPU shared
    // with other kernels, or more blocks than fit) join the count when they start, so warps
    // that ran out of work never wait for blocks that have not started.
    if (lane == 0) atomicAdd(&P.ctrl->active, 1u);
    __syncwarp();
    while (!(err & CSM_ERRBIT_TIMEOUT)) {
        if (deadline) {
            unsigned int late = 0;
            if (lane == 0) late = device_ns() > deadline;
            if (__shfl_sync(0xffffffffu, late, 0)) {
                err |= CSM_ERRBIT_TIMEOUT;
                break;
            }
        }
        int got = 0;
        if (have_source) {
            got = take_ticket(S, P);
            if (got < 0) continue;  // a frontier item that failed its check
            if (!got) have_source = false;
        }
        if (!got) got = claim_item(S, P);
        if (!got) {
            // Become idle: post one work request and wait (bounded) for donated work; leave
            // when no warp holds work and the ring is empty, withdrawing the request.
            if (lane == 0) {
                atomicSub(&P.ctrl->active, 1u);
                atomicAdd(&P.ctrl->hungry, 1u);
            }
            __syncwarp();
            bool resumed = false;
            for (uint32_t it = 0; it < P.idle_limit; it++) {
                if (claim_item(S, P)) {
                    if (lane == 0) atomicAdd(&P.ctrl->active, 1u);
                    __syncwarp();
                    resumed = true;
                    break;
                }
                unsigned int act = 0, qt = 0, qh = 0, late = 0;
                if (lane == 0) {
                    act = *(volatile unsigned int *)&P.ctrl->active;
                    qt = *(volatile unsigned int *)&P.ctrl->q_tail;
                    qh = *(volatile unsigned int *)&P.ctrl->q_head;
                    late = deadline && device_ns() > deadline;
                }
                act = __shfl_sync(0xffffffffu, act, 0);
                qt = __shfl_sync(0xffffffffu, qt, 0);
                qh = __shfl_sync(0xffffffffu, qh, 0);
                if (__shfl_sync(0xffffffffu, late, 0)) err |= CSM_ERRBIT_TIMEOUT;
                if ((act == 0 && qt >= qh) || (err & CSM_ERRBIT_TIMEOUT)) break;
                __nanosleep(512);
            }
            if (!resumed) {
                if (lane == 0) withdraw_request(P);
                __syncwarp();
                break;
            }
        }
        const unsigned long long c = run_item<LASTLOOP, MODE>(S, P, scans, probes, tails, shared, err, deadline);
        if (lane == 0 && c) atomicAdd(P.counts + S.item_plan, c);
        if ((scans | probes | tails | shared) >= (1u << 30)) {
            atomicAdd(&P.ctrl->scan_entries, (unsigned long long)scans);
            atomicAdd(&P.ctrl->probes, (unsigned long long)probes);
            // The tail and shared-level counters are warp-uniform: one lane adds them.
            if (lane == 0) atomicAdd(&P.ctrl->tail_lists, (unsigned long long)tails);
            if (lane == 0) atomicAdd(&P.ctrl->shared_last, (unsigned long long)shared);
            scans = probes = tails = shared = 0;
        }
        __syncwarp();
    }
    unsigned long long scans64 = scans, probes64 = probes;
    for (int o = 16; o > 0; o >>= 1) {
        scans64 += __shfl_xor_sync(0xffffffffu, scans64, o);
        probes64 += __shfl_xor_sync(0xffffffffu, probes64, o);
    }
    if (lane == 0) {
        if (scans64) atomicAdd(&P.ctrl->scan_entries, scans64);
        if (probes64) atomicAdd(&P.ctrl->probes, probes64);
        if (tails) atomicAdd(&P.ctrl->tail_lists, (unsigned long long)tails);
        if (shared) atomicAdd(&P.ctrl->shared_last, (unsigned long long)shared);
        if (err) atomicOr(&P.ctrl->error, err);
    }
}

// Per plan: the key range of its seed relation, and the number of 32-key seed chunks.
__global__ void k_seed_ranges(const DevPlan *plans, uint32_t nplans, const unsigned long long *keys, uint32_t m,
                              KeyLayout kl, uint32_t *seed_lo, uint32_t *chunks) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nplans) return;
    const uint32_t rel = plans[p].seed_rel;
    // [lo, hi) = keys whose relation field equals rel.
    uint32_t lo = 0, hi = m;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (kl.rel(keys[mid]) < rel) lo = mid + 1;
        else hi = mid;
    }
    uint32_t a = lo;
    lo = a;
    hi = m;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (kl.rel(keys[mid]) <= rel) lo = mid + 1;
        else hi = mid;
    }
    seed_lo[p] = a;
    seed_lo[nplans + p] = lo;
    chunks[p] = (lo - a + 31u) / 32u;
}

// Exclusive prefix of chunk counts (one block; plans are few).
__global__ void k_ticket_prefix(const uint32_t *chunks, uint32_t nplans, uint32_t *prefix, EnumControl *ctrl) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (nplans + blockDim.x - 1) / blockDim.x;
    uint32_t s = 0;
    for (uint32_t i = t * per; i < (t + 1) * per && i < nplans; i++) s += chunks[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        uint32_t acc = 0;
        for (uint32_t i = 0; i < blockDim.x; i++) {
            uint32_t v = part[i];
            part[i] = acc;
            acc += v;
        }
        ctrl->nticket = acc;
        prefix[nplans] = acc;
    }
    __syncthreads();
    uint32_t acc = part[t];
    for (uint32_t i = t * per; i < (t + 1) * per && i < nplans; i++) {
        prefix[i] = acc;
        acc += chunks[i];
    }
}

// Resets the control block for one launch.  The launch epoch (which marks queue slots ready)
// is the previous one plus one, kept on the device so that every launch on this scratch gets a
// fresh epoch whichever engine, stream or replayed graph issues it.
__global__ void k_ctrl_reset(EnumControl *ctrl, uint32_t active, unsigned long long nticket) {
    uint32_t epoch = ctrl->epoch + 1u;
    if (epoch == 0) epoch = 1;
    EnumControl c;
    memset(&c, 0, sizeof(c));
    c.active = active;
    c.epoch = epoch;
    c.nticket = nticket;
    c.t_start = device_ns();
    *ctrl = c;
}

// Upper bound of the next BFS level: sum over items of their smallest candidate list.
// Table of a pendant plan (DevPlan.memo_slot): for every data vertex v, the count of its
// counting level c for a prefix whose vertex at memo_depth is v — the candidates w of v's list
// under the flag rule and c's NLF filter, each with its Cartesian tail, exactly as the
// lane-parallel counting level sums them (no prefix exclusion can apply).  One warp per vertex.
__global__ void k_pendant_counts(EnumParams P, uint32_t plan, unsigned long long *out) {
    const uint32_t lane = threadIdx.x & 31u;
    const DevPlan *pl = P.plans + plan;
    const uint32_t c = pl->tail_start - 1u;
    const DevLevel *lv = &pl->lv[c];
    const uint32_t rel = __ldg(&lv->bn_rel[0]);
    const bool old = (__ldg(&lv->old_mask) & 1u) != 0;
    const uint32_t nlf_id = __ldg(&lv->nlf_bitmap);
    const uint32_t *nlf = nlf_id == CSM_NO_BITMAP ? nullptr : bitmap(P, nlf_id);
    uint32_t scans = 0, probes = 0, tails = 0;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    for (uint32_t v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); v < P.g.V; v += nw) {
        const uint2 ms = list_of(P, rel, v, 900 + c);
        unsigned long long acc = 0;
        for (uint32_t base = 0; base < ms.y; base += 32) {
            const uint32_t idx = base + lane;
            if (idx >= ms.y) continue;
            const uint32_t e = __ldg(P.g.pool + ms.x + idx);
            const uint32_t w = e >> 1;
            scans++;
            bool ok = !(old && (e & 1u));
            if (w >= P.g.V) {
                record_bad(P, CSM_BAD_ENTRY, e, ms.x + idx, 900 + c);
                ok = false;
            }
            if (ok && nlf) ok = test_bit(nlf, w);
            if (ok) {
                acc += tail_count_lane(nullptr, nullptr, P, pl, c, 0, w, 0, probes);
                tails++;
            }
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[v] = acc;
    }
    unsigned long long s64 = scans, p64 = probes, t64 = tails;
    for (int o = 16; o > 0; o >>= 1) {
        s64 += __shfl_xor_sync(0xffffffffu, s64, o);
        p64 += __shfl_xor_sync(0xffffffffu, p64, o);
        t64 += __shfl_xor_sync(0xffffffffu, t64, o);
    }
    if (lane == 0) {
        if (s64) atomicAdd(&P.ctrl->scan_entries, s64);
        if (p64) atomicAdd(&P.ctrl->probes, p64);
        if (t64) atomicAdd(&P.ctrl->tail_lists, t64);
    }
}

__global__ void k_expand_bound(EnumParams P, const WorkItem *items, const unsigned long long *nitems) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long nw = (unsigned long long)gridDim.x * (blockDim.x >> 5);
    const unsigned long long n = *nitems;
    unsigned long long acc = 0;
    for (unsigned long long i = (blockIdx.x * (blockDim.x >> 5)) + (threadIdx.x >> 5); i < n; i += nw) {
        const WorkItem *it = items + i;
        const DevPlan *pl = P.plans + it->plan;
        const uint32_t d = it->depth;
        if (d >= pl->expand_stop) {
            if (lane == 0) acc += 1;  // passes through unchanged
            continue;
        }
        const DevLevel *lv = &pl->lv[d];
        uint32_t sz = 0xFFFFFFFFu;
        if (lane < lv->nbn) {
            sz = list_of(P, lv->bn_rel[lane], it->f[lv->bn_depth[lane]], 800 + d).y;
        }
        for (int o = 16; o > 0; o >>= 1) sz = min(sz, __shfl_xor_sync(0xffffffffu, sz, o));
        if (lane == 0) acc += sz;
    }
    if (lane == 0 && acc) atomicAdd(&P.ctrl->expand_bound, acc);
}

}  // namespace

size_t enum_smem_bytes(int warps_per_block) { return sizeof(WarpState) * (size_t)warps_per_block; }

namespace {
using EnumKernel = void (*)(EnumParams);
template <int MINB>
EnumKernel enum_kernel_mode(bool last_loop, uint32_t mode) {
    if (mode == CSM_ENUM_MODE_EXPAND) return k_enumerate<MINB, false, CSM_ENUM_MODE_EXPAND>;
    if (mode == CSM_ENUM_MODE_ROWS) return k_enumerate<MINB, false, CSM_ENUM_MODE_ROWS>;
    return last_loop ? k_enumerate<MINB, true, CSM_ENUM_MODE_COUNT> : k_enumerate<MINB, false, CSM_ENUM_MODE_COUNT>;
}

EnumKernel enum_kernel(int occupancy, bool last_loop, uint32_t mode) {
    switch (occupancy) {
        case 6: return enum_kernel_mode<6>(last_loop, mode);
        case 5: return enum_kernel_mode<5>(last_loop, mode);
        default: return enum_kernel_mode<4>(last_loop, mode);
    }
}
}  // namespace

int enum_blocks_per_sm(int warps_per_block, int occupancy) {
    // The smallest residency of the variants: a persistent grid must fit each of them.
    const size_t smem = enum_smem_bytes(warps_per_block);
    int best = 1 << 30;
    for (int v = 0; v < 4; v++) {
        EnumKernel k = enum_kernel(occupancy, v == 1, v < 2 ? CSM_ENUM_MODE_COUNT : (uint32_t)(v - 1));
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, warps_per_block * 32, smem) != cudaSuccess) return 1;
        best = nb < best ? nb : best;
    }
    return best > 0 ? best : 1;
}

void launch_enumerate(const EnumParams &p, int blocks, int warps_per_block, int occupancy, cudaStream_t s) {
    const size_t smem = enum_smem_bytes(warps_per_block);
    EnumKernel k = enum_kernel(occupancy, p.last_loop != 0, p.mode);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<blocks, warps_per_block * 32, smem, s>>>(p);
}

void launch_seed_tickets(const DevPlan *plans, uint32_t nplans, const unsigned long long *keys, uint32_t m,
                         KeyLayout kl, uint32_t *seed_lo, uint32_t *ticket_prefix, EnumControl *ctrl,
                         cudaStream_t s) {
    // seed_lo holds three arrays of nplans: first key, end key, chunk count.
    uint32_t *chunks = seed_lo + 2 * nplans;
    k_seed_ranges<<<(nplans + 127) / 128, 128, 0, s>>>(plans, nplans, keys, m, kl, seed_lo, chunks);
    k_ticket_prefix<<<1, 1024, 0, s>>>(chunks, nplans, ticket_prefix, ctrl);
}

void launch_ctrl_reset(EnumControl *ctrl, uint32_t active, unsigned long long nticket, cudaStream_t s) {
    k_ctrl_reset<<<1, 1, 0, s>>>(ctrl, active, nticket);
}

void launch_pendant_counts(const EnumParams &p, uint32_t plan, unsigned long long *out, cudaStream_t s) {
    k_pendant_counts<<<148 * 8, 256, 0, s>>>(p, plan, out);
}

void launch_expand_bound(const EnumParams &p, const WorkItem *items, const unsigned long long *nitems,
                         cudaStream_t s) {
    k_expand_bound<<<296, 256, 0, s>>>(p, items, nitems);
}

}  // namespace csm
