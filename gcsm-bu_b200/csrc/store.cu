// Device graph store: building the label-partitioned CSR with slack, applying a batch of
// insertions and deletions, and keeping the NLF candidate bitmaps current.
//
// Replaces the reference's BuildTriesFromEdgeList (graph/match_gpu.cu:2296-2344),
// AllocRelation + setCapacities/roundCapacities/setNeighborPointers (match_gpu.cu:2346-2417,
// kernels/indexing.cu:12-74), addTriesToGraph (indexing.cu:76-263) and the candidate part of
// UpdateGlobalIndex / getGlobalCandidates (match_gpu.cu:611-834, indexing.cu:303-337).
//
// A batch is turned into 64-bit keys (relation, src, dst, op), one per orientation that a
// query edge can take, sorted, and classified against the current lists.  The keys of one
// adjacency list form one contiguous segment, so every list touched by the batch is handled
// by one warp: deletions are compacted out, insertions are merged in place from the back
// (or into a fresh slack segment when the list is full).
#include <algorithm>
#include <cub/cub.cuh>

#include "kernels.cuh"
#include "store.cuh"

namespace csm {

namespace {

__device__ __forceinline__ uint32_t slack_capacity(uint32_t size) {
    // max(8, 2^(ceil(log2 size) + 1)), the rounding of indexing.cu:46-59 in integer form.
    if (size == 0) return 0;
    uint32_t p = size <= 1 ? 1u : 1u << (32 - __clz(size - 1));
    uint64_t c = (uint64_t)p * 2;
    if (c < 8) c = 8;
    return c > 0x80000000ull ? 0x80000000u : (uint32_t)c;
}

__global__ void k_build_keys(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elab,
                             const uint8_t *isdel, uint32_t V, const uint8_t *vlab, const uint32_t *elab_raw,
                             uint32_t nel, const uint16_t *rel_table, uint32_t nvl, KeyLayout kl,
                             unsigned long long *keys) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = src[i], y = dst[i];
        unsigned long long k0 = CSM_INVALID_KEY, k1 = CSM_INVALID_KEY;
        if (x < V && y < V && x != y) {
            const uint32_t a = vlab[x], b = vlab[y];
            if (a != CSM_NO_LABEL && b != CSM_NO_LABEL) {
                const uint32_t lr = elab[i];
                uint32_t lo = 0, hi = nel;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (elab_raw[mid] < lr) lo = mid + 1;
                    else hi = mid;
                }
                if (lo < nel && elab_raw[lo] == lr) {
                    const uint32_t op = (isdel && isdel[i]) ? 1u : 0u;
                    const uint32_t r1 = rel_table[((size_t)a * nel + lo) * nvl + b];
                    const uint32_t r2 = rel_table[((size_t)b * nel + lo) * nvl + a];
                    if (r1 != CSM_NO_REL) k0 = kl.make(r1, x, y, op);
                    if (r2 != CSM_NO_REL) k1 = kl.make(r2, y, x, op);
                }
            }
        }
        keys[2 * i] = k0;
        keys[2 * i + 1] = k1;
    }
}

// Deduplicates and classifies sorted keys; marks the entries of effective deletions and
// collects the first key of every adjacency-list segment.
__global__ void k_classify(uint32_t m, const unsigned long long *keys, KeyLayout kl, const uint2 *meta,
                           uint32_t *pool, uint32_t V, uint8_t *eff, uint32_t *heads, unsigned int *nheads,
                           unsigned long long *counters) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[p];
        uint8_t e = CSM_EFF_NONE;
        if (k != CSM_INVALID_KEY) {
            const unsigned long long prev = p ? keys[p - 1] : CSM_INVALID_KEY;
            if (p == 0 || kl.list_of(prev) != kl.list_of(k)) heads[atomicAdd(nheads, 1u)] = p;
            if (p == 0 || (prev >> 1) != (k >> 1)) {
                const uint32_t r = kl.rel(k), x = kl.src(k), y = kl.dst(k);
                const uint2 ms = meta[(size_t)r * V + x];
                const uint32_t *list = pool + ms.x;
                uint32_t lo = 0, hi = ms.y;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (list[mid] < (y << 1)) lo = mid + 1;
                    else hi = mid;
                }
                const bool found = lo < ms.y && (list[lo] >> 1) == y;
                if ((k & 1ull) == 0) {
                    e = found ? CSM_EFF_NONE : CSM_EFF_INS;
                } else if (found) {
                    e = CSM_EFF_DEL;
                    pool[ms.x + lo] = (y << 1) | 1u;
                }
                if (e != CSM_EFF_NONE && x < y) atomicAdd(counters + (e - 1), 1ull);
            }
        }
        eff[p] = e;
    }
}

// Per segment: end position and the number of effective insertions and deletions.
__global__ void k_seg_info(const uint32_t *heads, const unsigned int *nheads, const unsigned long long *keys,
                           uint32_t m, KeyLayout kl, const uint8_t *eff, uint32_t *seg_nins, uint32_t *seg_ndel,
                           uint32_t *seg_end) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    const uint32_t nh = *nheads;
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nh; i += nw) {
        const uint32_t h = heads[i];
        const unsigned long long lk = kl.list_of(keys[h]);
        uint32_t ni = 0, nd = 0, end = h;
        for (uint32_t base = h;; base += 32) {
            const uint32_t p = base + lane;
            const bool in = p < m && keys[p] != CSM_INVALID_KEY && kl.list_of(keys[p]) == lk;
            const uint8_t e = in ? eff[p] : 0;
            ni += __popc(__ballot_sync(0xffffffffu, e == CSM_EFF_INS));
            nd += __popc(__ballot_sync(0xffffffffu, e == CSM_EFF_DEL));
            const uint32_t inm = __ballot_sync(0xffffffffu, in);
            if (inm != 0xffffffffu) {
                end = base + __popc(inm);
                break;
            }
        }
        if (lane == 0) {
            seg_nins[h] = ni;
            seg_ndel[h] = nd;
            seg_end[h] = end;
        }
    }
}

// Removes the flagged (deleted) entries of every list with deletions.
__global__ void k_del_compact(const uint32_t *heads, const unsigned int *nheads, const unsigned long long *keys,
                              KeyLayout kl, const uint32_t *seg_ndel, uint2 *meta, uint32_t *pool, uint32_t V) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    const uint32_t nh = *nheads;
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nh; i += nw) {
        const uint32_t h = heads[i];
        if (seg_ndel[h] == 0) continue;
        const unsigned long long k = keys[h];
        const size_t mi = (size_t)kl.rel(k) * V + kl.src(k);
        const uint2 ms = meta[mi];
        uint32_t w = 0;
        for (uint32_t base = 0; base < ms.y; base += 32) {
            const uint32_t idx = base + lane;
            const uint32_t e = idx < ms.y ? pool[ms.x + idx] : 1u;
            const bool keep = idx < ms.y && !(e & 1u);
            const uint32_t mask = __ballot_sync(0xffffffffu, keep);
            if (keep) pool[ms.x + w + __popc(mask & ((1u << lane) - 1u))] = e;
            w += __popc(mask);
            __syncwarp();
        }
        if (lane == 0) meta[mi].y = w;
    }
}

// Merges the effective insertions of every touched list, flagged, keeping lists sorted.
// scr_y / scr_lb (indexed by segment position) receive the inserted ids and, for each, the
// number of old entries below it; the final position of insertion j is scr_lb + j.
__global__ void k_ins_merge(const uint32_t *heads, const unsigned int *nheads, const unsigned long long *keys,
                            KeyLayout kl, const uint8_t *eff, const uint32_t *seg_nins, const uint32_t *seg_end,
                            uint2 *meta, uint32_t *cap, uint32_t *pool, uint32_t V, unsigned long long *pool_top,
                            unsigned long long pool_cap, uint32_t *scr_y, uint32_t *scr_lb, unsigned int *error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    const uint32_t nh = *nheads;
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nh; i += nw) {
        const uint32_t h = heads[i];
        const uint32_t k = seg_nins[h];
        if (k == 0) continue;
        const unsigned long long key = keys[h];
        const size_t mi = (size_t)kl.rel(key) * V + kl.src(key);
        const uint2 ms = meta[mi];
        const uint32_t d = ms.y, c = cap[mi];
        const uint32_t *A = pool + ms.x;
        const uint32_t end = seg_end[h];
        // A rerun after a pool overflow skips lists that were already merged (all or none of
        // a list's insertions are applied, so checking the first one suffices).
        {
            bool merged = false;
            if (lane == 0) {
                uint32_t p = h;
                while (p < end && eff[p] != CSM_EFF_INS) p++;
                const uint32_t y = kl.dst(keys[p]);
                uint32_t lo = 0, hi = d;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (A[mid] < (y << 1)) lo = mid + 1;
                    else hi = mid;
                }
                merged = lo < d && (A[lo] >> 1) == y;
            }
            if (__shfl_sync(0xffffffffu, merged, 0)) continue;
        }
        // Phase A: compact the inserted ids and their ranks among the old entries.
        uint32_t j = 0;
        for (uint32_t base = h; base < end; base += 32) {
            const uint32_t p = base + lane;
            const bool ins = p < end && eff[p] == CSM_EFF_INS;
            const uint32_t mask = __ballot_sync(0xffffffffu, ins);
            if (ins) {
                const uint32_t y = kl.dst(keys[p]);
                uint32_t lo = 0, hi = d;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (A[mid] < (y << 1)) lo = mid + 1;
                    else hi = mid;
                }
                const uint32_t jj = j + __popc(mask & ((1u << lane) - 1u));
                scr_y[h + jj] = y;
                scr_lb[h + jj] = lo;
            }
            j += __popc(mask);
        }
        __syncwarp();
        uint32_t dst_off = ms.x;
        const bool relocate = d + k > c;
        if (relocate) {
            uint32_t need = d + k;
            uint32_t p2 = 1u << (32 - __clz(need - 1 | 1u));
            unsigned long long nc = (unsigned long long)p2 * 2;
            if (nc < 8) nc = 8;
            unsigned long long off = 0;
            if (lane == 0) off = atomicAdd(pool_top, nc);
            off = __shfl_sync(0xffffffffu, off, 0);
            if (off + nc > pool_cap || off + nc > 0xFFFFFFFFull) {
                if (lane == 0) atomicOr(error, CSM_ERRBIT_POOL);
                continue;
            }
            dst_off = (uint32_t)off;
            if (lane == 0) cap[mi] = (uint32_t)nc;
        }
        // Phase B: move the old entries right by the number of insertions below them.
        const uint32_t *LB = scr_lb + h;
        const uint32_t first = relocate ? 0u : LB[0];
        for (int32_t t = (int32_t)d; t > (int32_t)first; t -= 32) {
            const int32_t s = t - 32 > (int32_t)first ? t - 32 : (int32_t)first;
            const int32_t ii = s + (int32_t)lane;
            uint32_t a = 0, dest = 0;
            const bool act = ii < t;
            if (act) {
                a = pool[ms.x + ii];
                // shift = #{j : LB[j] <= ii}
                uint32_t lo = 0, hi = k;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (LB[mid] <= (uint32_t)ii) lo = mid + 1;
                    else hi = mid;
                }
                dest = (uint32_t)ii + lo;
            }
            __syncwarp();
            if (act) pool[dst_off + dest] = a;
            __syncwarp();
        }
        // Phase C: write the insertions, flagged.
        for (uint32_t jj = lane; jj < k; jj += 32) pool[dst_off + LB[jj] + jj] = (scr_y[h + jj] << 1) | 1u;
        __syncwarp();
        if (lane == 0) meta[mi] = make_uint2(dst_off, d + k);
    }
}

// Clears the flags of this batch's insertions.
__global__ void k_clear_ins(const uint32_t *heads, const unsigned int *nheads, const unsigned long long *keys,
                            KeyLayout kl, const uint32_t *seg_nins, const uint2 *meta, uint32_t *pool, uint32_t V,
                            const uint32_t *scr_lb, const unsigned int *error) {
    // After a failed merge some lists were not merged; the batch is redone, so clear nothing.
    if (*(volatile const unsigned int *)error & CSM_ERRBIT_POOL) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    const uint32_t nh = *nheads;
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nh; i += nw) {
        const uint32_t h = heads[i];
        const uint32_t k = seg_nins[h];
        if (k == 0) continue;
        const unsigned long long key = keys[h];
        const uint2 ms = meta[(size_t)kl.rel(key) * V + kl.src(key)];
        for (uint32_t jj = lane; jj < k; jj += 32) pool[ms.x + scr_lb[h + jj] + jj] &= ~1u;
    }
}

__device__ __forceinline__ void refresh_nlf(uint32_t x, uint32_t a, const uint2 *meta, uint32_t V,
                                            const uint32_t *spec_begin, const NlfSpec *specs, uint32_t *bits,
                                            uint32_t words) {
    for (uint32_t s = spec_begin[a]; s < spec_begin[a + 1]; s++) {
        const NlfSpec &sp = specs[s];
        bool pass = true;
        for (uint32_t g = 0; g < sp.ngroups && pass; g++) pass = meta[(size_t)sp.rel[g] * V + x].y >= sp.cnt[g];
        uint32_t *w = bits + (size_t)sp.bitmap * words + (x >> 5);
        const uint32_t bit = 1u << (x & 31);
        if (pass) atomicOr(w, bit);
        else atomicAnd(w, ~bit);
    }
}

// NLF refresh for the source vertex of every list the batch changed.
__global__ void k_nlf_update(const uint32_t *heads, const unsigned int *nheads, const unsigned long long *keys,
                             KeyLayout kl, const uint32_t *seg_nins, const uint32_t *seg_ndel, const uint2 *meta,
                             uint32_t V, const uint8_t *vlab, const uint32_t *spec_begin, const NlfSpec *specs,
                             uint32_t *bits, uint32_t words) {
    const uint32_t nh = *nheads;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
        const uint32_t h = heads[i];
        if (seg_nins[h] == 0 && seg_ndel[h] == 0) continue;
        const uint32_t x = kl.src(keys[h]);
        refresh_nlf(x, vlab[x], meta, V, spec_begin, specs, bits, words);
    }
}

__global__ void k_nlf_all(uint32_t V, const uint8_t *vlab, const uint2 *meta, const uint32_t *spec_begin,
                          const NlfSpec *specs, uint32_t *bits, uint32_t words) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < V; x += gridDim.x * blockDim.x) {
        const uint32_t a = vlab[x];
        if (a == CSM_NO_LABEL) continue;
        refresh_nlf(x, a, meta, V, spec_begin, specs, bits, words);
    }
}

// Initial build: unique sorted keys -> list sizes, capacities, entries.
__global__ void k_mark_unique(uint32_t m, const unsigned long long *keys, uint8_t *flag) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[p];
        flag[p] = k != CSM_INVALID_KEY && (p == 0 || (keys[p - 1] >> 1) != (k >> 1));
    }
}

__global__ void k_list_sizes(uint32_t mu, const unsigned long long *ukeys, KeyLayout kl, uint2 *meta, uint32_t *cap,
                             uint32_t V) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < mu; p += gridDim.x * blockDim.x) {
        const unsigned long long k = ukeys[p];
        if (p > 0 && kl.list_of(ukeys[p - 1]) == kl.list_of(k)) continue;
        const unsigned long long lk = kl.list_of(k);
        uint32_t lo = p, hi = mu;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (kl.list_of(ukeys[mid]) <= lk) lo = mid + 1;
            else hi = mid;
        }
        const size_t mi = (size_t)kl.rel(k) * V + kl.src(k);
        meta[mi].y = lo - p;
        cap[mi] = slack_capacity(lo - p);
    }
}

__global__ void k_set_offsets(size_t n, const unsigned long long *off, uint2 *meta) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        meta[i].x = (uint32_t)off[i];
}

__global__ void k_scatter(uint32_t mu, const unsigned long long *ukeys, KeyLayout kl, const uint2 *meta, uint32_t *pool,
                          uint32_t V) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < mu; p += gridDim.x * blockDim.x) {
        const unsigned long long k = ukeys[p];
        const unsigned long long lk = kl.list_of(k);
        uint32_t lo = 0, hi = p;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (kl.list_of(ukeys[mid]) < lk) lo = mid + 1;
            else hi = mid;
        }
        const uint2 ms = meta[(size_t)kl.rel(k) * V + kl.src(k)];
        pool[ms.x + (p - lo)] = kl.dst(k) << 1;
    }
}

// Compaction: the fresh-slack capacity of every list (from its size), as 64-bit values to be
// prefix-summed into the new layout's offsets.  Nothing of the current layout changes.
__global__ void k_fresh_caps(size_t n, const uint2 *meta, unsigned long long *cap64) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        cap64[i] = slack_capacity(meta[i].y);
}

// Compaction commit: capacities of the new layout.
__global__ void k_set_caps(size_t n, const uint2 *meta, uint32_t *cap) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        cap[i] = slack_capacity(meta[i].y);
}

__global__ void k_copy_lists(size_t n, const uint2 *meta, const unsigned long long *newoff, const uint32_t *src,
                             uint32_t *dst) {
    const uint32_t lane = threadIdx.x & 31u;
    const size_t nw = (size_t)gridDim.x * (blockDim.x >> 5);
    for (size_t i = blockIdx.x * (size_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nw) {
        const uint2 ms = meta[i];
        for (uint32_t j = lane; j < ms.y; j += 32) dst[newoff[i] + j] = src[ms.x + j];
    }
}

__global__ void k_u32_to_u64(size_t n, const uint32_t *a, unsigned long long *b) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

// Planner statistics per directed query edge: candidate edges and sources with >= 1 of them.
__global__ void k_edge_stats(uint32_t V, const uint2 *meta, const uint32_t *pool, uint32_t rel, const uint32_t *bits_u,
                             const uint32_t *bits_uu, unsigned long long *out) {
    unsigned long long sum = 0, srcs = 0;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < V; x += gridDim.x * blockDim.x) {
        if (!((bits_u[x >> 5] >> (x & 31)) & 1u)) continue;
        const uint2 ms = meta[(size_t)rel * V + x];
        uint32_t c = 0;
        for (uint32_t j = 0; j < ms.y; j++) {
            const uint32_t w = pool[ms.x + j] >> 1;
            c += (bits_uu[w >> 5] >> (w & 31)) & 1u;
        }
        sum += c;
        srcs += c ? 1 : 0;
    }
    if (sum) atomicAdd(out, sum);
    if (srcs) atomicAdd(out + 1, srcs);
}

// Net change of each relation's entry count in this batch (+1 per effective insertion, -1 per
// effective deletion, per key orientation).  Keys are sorted by relation, so the lanes of a warp
// mostly share one relation: each group of equal relations adds its sum once.
__global__ void k_rel_delta(uint32_t m, const unsigned long long *keys, KeyLayout kl, const uint8_t *eff,
                            long long *delta) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < m;
    const uint32_t rel = in ? kl.rel(keys[i]) : 0xFFFFFFFFu;
    const uint8_t e = in ? eff[i] : CSM_EFF_NONE;
    int v = e == CSM_EFF_INS ? 1 : (e == CSM_EFF_DEL ? -1 : 0);
    const uint32_t group = __match_any_sync(0xffffffffu, rel);
    int sum = 0;
    for (uint32_t g = group; g; g &= g - 1) sum += __shfl_sync(group, v, __ffs(g) - 1);
    if (in && sum != 0 && (threadIdx.x & 31u) == (uint32_t)(__ffs(group) - 1))
        atomicAdd(reinterpret_cast<unsigned long long *>(delta + rel), (unsigned long long)(long long)sum);  // two's complement
}

// Bit per vertex that owns a list some batch key belongs to (the key's source).  Keys are
// sorted, so neighbouring lanes mostly share a word; one lane per distinct source sets it.
// Updates that match no relation carry CSM_INVALID_KEY (sorted to the end): they own no list,
// and their all-ones source field is no vertex, so they are skipped.
__global__ void k_touched(uint32_t m, const unsigned long long *keys, KeyLayout kl, uint32_t *bits, uint32_t words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const unsigned long long k = keys[i];
    if (k == CSM_INVALID_KEY) return;
    const uint32_t x = kl.src(k);
    if (i > 0 && kl.src(keys[i - 1]) == x) return;
    if ((x >> 5) < words) atomicOr(bits + (x >> 5), 1u << (x & 31));
}

// Entry count of every relation (sum of its list sizes).  The loop is warp-uniform so that all
// lanes take part in the grouping shuffles.
__global__ void k_rel_sizes(uint32_t V, uint32_t R, const uint2 *meta, unsigned long long *out) {
    const size_t total = (size_t)V * R;
    const uint32_t lane = threadIdx.x & 31u;
    const size_t warps = (size_t)gridDim.x * (blockDim.x >> 5);
    for (size_t w = (size_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < total; w += warps) {
        const size_t i = w * 32 + lane;
        const bool in = i < total;
        const uint32_t rel = in ? (uint32_t)(i / V) : 0xFFFFFFFFu;
        const uint32_t sz = in ? meta[i].y : 0u;
        const uint32_t group = __match_any_sync(0xffffffffu, rel);
        unsigned long long sum = 0;
        for (uint32_t g = group; g; g &= g - 1) sum += __shfl_sync(group, sz, __ffs(g) - 1);
        if (in && lane == (uint32_t)(__ffs(group) - 1) && sum) atomicAdd(out + rel, sum);
    }
}

inline int grid_for(size_t n, int block) {
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 16) g = 148 * 16;
    return (int)g;
}

}  // namespace

void store_build_keys(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elab, const uint8_t *isdel,
                      const LabelTables &lt, const DeviceGraph &g, KeyLayout kl, unsigned long long *keys,
                      cudaStream_t s) {
    k_build_keys<<<grid_for(n, 256), 256, 0, s>>>(n, src, dst, elab, isdel, g.V, g.vlab, lt.elab_raw, lt.nel,
                                                  lt.rel_table, lt.nvl, kl, keys);
}

cudaError_t store_sort_keys(void *temp, size_t &temp_bytes, const unsigned long long *in, unsigned long long *out,
                            uint32_t m, KeyLayout kl, cudaStream_t s) {
    return cub::DeviceRadixSort::SortKeys(temp, temp_bytes, in, out, (int)m, 0, (int)kl.end_bit(), s);
}

void store_classify(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                    cudaStream_t s) {
    k_classify<<<grid_for(m, 256), 256, 0, s>>>(m, keys, kl, g.meta, g.pool, g.V, b.eff, b.heads, b.nheads,
                                                b.counters);
    k_seg_info<<<grid_for((size_t)m * 32, 256), 256, 0, s>>>(b.heads, b.nheads, keys, m, kl, b.eff, b.seg_nins,
                                                             b.seg_ndel, b.seg_end);
}

void store_delete(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                  cudaStream_t s) {
    k_del_compact<<<grid_for((size_t)m * 32, 256), 256, 0, s>>>(b.heads, b.nheads, keys, kl, b.seg_ndel, g.meta,
                                                                g.pool, g.V);
}

void store_insert(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                  cudaStream_t s) {
    k_ins_merge<<<grid_for((size_t)m * 32, 256), 256, 0, s>>>(b.heads, b.nheads, keys, kl, b.eff, b.seg_nins,
                                                              b.seg_end, g.meta, g.cap, g.pool, g.V, g.pool_top,
                                                              g.pool_cap, b.scr_y, b.scr_lb, b.error);
}

void store_nlf_update(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                      const NlfTables &nt, cudaStream_t s) {
    k_nlf_update<<<grid_for(m, 256), 256, 0, s>>>(b.heads, b.nheads, keys, kl, b.seg_nins, b.seg_ndel, g.meta, g.V,
                                                  g.vlab, nt.spec_begin, nt.specs, nt.bits, nt.words);
}

void store_clear_ins(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                     cudaStream_t s) {
    k_clear_ins<<<grid_for((size_t)m * 32, 256), 256, 0, s>>>(b.heads, b.nheads, keys, kl, b.seg_nins, g.meta, g.pool,
                                                              g.V, b.scr_lb, b.error);
}

void store_nlf_all(DeviceGraph &g, const NlfTables &nt, cudaStream_t s) {
    k_nlf_all<<<grid_for(g.V, 256), 256, 0, s>>>(g.V, g.vlab, g.meta, nt.spec_begin, nt.specs, nt.bits, nt.words);
}

void store_rel_delta(uint32_t m, const unsigned long long *keys, KeyLayout kl, const BatchScratch &b, long long *delta,
                     cudaStream_t s) {
    if (m) k_rel_delta<<<(m + 255) / 256, 256, 0, s>>>(m, keys, kl, b.eff, delta);
}

void store_touched(uint32_t m, const unsigned long long *keys, KeyLayout kl, uint32_t *bits, uint32_t words,
                   cudaStream_t s) {
    cudaMemsetAsync(bits, 0, sizeof(uint32_t) * words, s);
    if (m) k_touched<<<(m + 255) / 256, 256, 0, s>>>(m, keys, kl, bits, words);
}

void store_rel_sizes(const DeviceGraph &g, unsigned long long *out, cudaStream_t s) {
    k_rel_sizes<<<grid_for((size_t)g.V * g.R, 256), 256, 0, s>>>(g.V, g.R, g.meta, out);
}

void store_edge_stats(DeviceGraph &g, uint32_t rel, const uint32_t *bits_u, const uint32_t *bits_uu,
                      unsigned long long *out, cudaStream_t s) {
    k_edge_stats<<<grid_for(g.V, 256), 256, 0, s>>>(g.V, g.meta, g.pool, rel, bits_u, bits_uu, out);
}

// Builds all lists from unique sorted keys.  Returns the total capacity (entries) laid out.
cudaError_t store_build_from_keys(DeviceGraph &g, const unsigned long long *keys_sorted, uint32_t m, KeyLayout kl,
                                  cudaStream_t s, std::string &err) {
    const size_t nmeta = (size_t)g.R * g.V;
    uint8_t *flag = nullptr;
    unsigned long long *ukeys = nullptr, *cap64 = nullptr;
    int *nsel = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
    cudaError_t e = cudaSuccess;
#define CSM_TRY(x)                      \
    do {                                \
        e = (x);                        \
        if (e != cudaSuccess) goto done; \
    } while (0)
    {
        CSM_TRY(cudaMalloc(&flag, (size_t)m + 1));
        CSM_TRY(cudaMalloc(&ukeys, sizeof(unsigned long long) * ((size_t)m + 1)));
        CSM_TRY(cudaMalloc(&nsel, sizeof(int)));
        CSM_TRY(cudaMalloc(&cap64, sizeof(unsigned long long) * (nmeta + 1)));
        k_mark_unique<<<grid_for(m, 256), 256, 0, s>>>(m, keys_sorted, flag);
        CSM_TRY(cub::DeviceSelect::Flagged(nullptr, temp_bytes, keys_sorted, flag, ukeys, nsel, (int)m, s));
        size_t tb2 = 0;
        CSM_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb2, cap64, cap64, nmeta + 1, s));
        temp_bytes = std::max(temp_bytes, tb2);
        CSM_TRY(cudaMalloc(&temp, temp_bytes + 16));
        CSM_TRY(cub::DeviceSelect::Flagged(temp, temp_bytes, keys_sorted, flag, ukeys, nsel, (int)m, s));
        int mu = 0;
        CSM_TRY(cudaMemcpyAsync(&mu, nsel, sizeof(int), cudaMemcpyDeviceToHost, s));
        CSM_TRY(cudaStreamSynchronize(s));
        CSM_TRY(cudaMemsetAsync(g.meta, 0, sizeof(uint2) * nmeta, s));
        CSM_TRY(cudaMemsetAsync(g.cap, 0, sizeof(uint32_t) * nmeta, s));
        if (mu > 0) k_list_sizes<<<grid_for(mu, 256), 256, 0, s>>>((uint32_t)mu, ukeys, kl, g.meta, g.cap, g.V);
        k_u32_to_u64<<<grid_for(nmeta, 256), 256, 0, s>>>(nmeta, g.cap, cap64);
        CSM_TRY(cudaMemsetAsync(cap64 + nmeta, 0, sizeof(unsigned long long), s));
        CSM_TRY(cub::DeviceScan::ExclusiveSum(temp, temp_bytes, cap64, cap64, nmeta + 1, s));
        unsigned long long total = 0;
        CSM_TRY(cudaMemcpyAsync(&total, cap64 + nmeta, sizeof(total), cudaMemcpyDeviceToHost, s));
        CSM_TRY(cudaStreamSynchronize(s));
        if (total > g.pool_cap) {
            err = "adjacency pool too small for the initial graph";
            e = cudaErrorMemoryAllocation;
            goto done;
        }
        k_set_offsets<<<grid_for(nmeta, 256), 256, 0, s>>>(nmeta, cap64, g.meta);
        if (mu > 0) k_scatter<<<grid_for(mu, 256), 256, 0, s>>>((uint32_t)mu, ukeys, kl, g.meta, g.pool, g.V);
        CSM_TRY(cudaMemcpyAsync(g.pool_top, &total, sizeof(total), cudaMemcpyHostToDevice, s));
        CSM_TRY(cudaStreamSynchronize(s));
        CSM_TRY(cudaGetLastError());
    }
done:
    cudaFree(flag);
    cudaFree(ukeys);
    cudaFree(nsel);
    cudaFree(cap64);
    cudaFree(temp);
    return e;
#undef CSM_TRY
}

// Layout of a compaction, without changing the graph: `offsets` (nmeta + 1 entries, allocated
// here; release with cudaFree) receives every list's offset in a fresh-slack layout, and `total`
// the entries that layout needs.
cudaError_t store_layout(const DeviceGraph &g, unsigned long long **offsets, unsigned long long &total, cudaStream_t s) {
    const size_t nmeta = (size_t)g.R * g.V;
    unsigned long long *cap64 = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
    *offsets = nullptr;
    cudaError_t e = cudaMalloc(&cap64, sizeof(unsigned long long) * (nmeta + 1));
    if (e != cudaSuccess) return e;
    k_fresh_caps<<<grid_for(nmeta, 256), 256, 0, s>>>(nmeta, g.meta, cap64);
    if ((e = cudaMemsetAsync(cap64 + nmeta, 0, sizeof(unsigned long long), s)) == cudaSuccess &&
        (e = cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, cap64, cap64, nmeta + 1, s)) == cudaSuccess &&
        (e = cudaMalloc(&temp, temp_bytes + 16)) == cudaSuccess &&
        (e = cub::DeviceScan::ExclusiveSum(temp, temp_bytes, cap64, cap64, nmeta + 1, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(&total, cap64 + nmeta, sizeof(total), cudaMemcpyDeviceToHost, s)) == cudaSuccess)
        e = cudaStreamSynchronize(s);
    cudaFree(temp);
    if (e != cudaSuccess) {
        cudaFree(cap64);
        return e;
    }
    *offsets = cap64;
    return cudaGetLastError();
}

// Moves every list to `offsets` (from store_layout) inside `new_pool` and makes that layout the
// graph's: offsets, capacities and the bump pointer.  The caller then swaps the pools.
cudaError_t store_relayout(DeviceGraph &g, uint32_t *new_pool, const unsigned long long *offsets,
                           unsigned long long total, cudaStream_t s) {
    const size_t nmeta = (size_t)g.R * g.V;
    k_copy_lists<<<grid_for(nmeta * 32, 256), 256, 0, s>>>(nmeta, g.meta, offsets, g.pool, new_pool);
    k_set_offsets<<<grid_for(nmeta, 256), 256, 0, s>>>(nmeta, offsets, g.meta);
    k_set_caps<<<grid_for(nmeta, 256), 256, 0, s>>>(nmeta, g.meta, g.cap);
    cudaError_t e = cudaMemcpyAsync(g.pool_top, &total, sizeof(total), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace csm
