// Device helpers and kernel declarations shared by the engine's .cu files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.h"

namespace csm {

// Layout of the 64-bit batch keys: [rel | src | dst | op], op 0 = insert, 1 = delete.
struct KeyLayout {
    uint32_t vbits;   // bits per vertex id
    uint32_t rbits;   // bits per relation id
    __host__ __device__ unsigned long long make(uint32_t rel, uint32_t x, uint32_t y, uint32_t op) const {
        return ((unsigned long long)rel << (2 * vbits + 1)) | ((unsigned long long)x << (vbits + 1)) |
               ((unsigned long long)y << 1) | (unsigned long long)op;
    }
    __host__ __device__ uint32_t rel(unsigned long long k) const { return (uint32_t)(k >> (2 * vbits + 1)); }
    __host__ __device__ uint32_t src(unsigned long long k) const {
        return (uint32_t)((k >> (vbits + 1)) & ((1ull << vbits) - 1));
    }
    __host__ __device__ uint32_t dst(unsigned long long k) const { return (uint32_t)((k >> 1) & ((1ull << vbits) - 1)); }
    // (rel, src) part, used to find the segment of one adjacency list.
    __host__ __device__ unsigned long long list_of(unsigned long long k) const { return k >> (vbits + 1); }
    __host__ __device__ unsigned long long list_key(uint32_t rel, uint32_t x) const {
        return ((unsigned long long)rel << vbits) | x;
    }
    __host__ __device__ uint32_t end_bit() const { return rbits + 2 * vbits + 1; }
};

// Read-only view of the device graph used by every kernel.
struct GraphView {
    const uint2 *meta;       // [R * V] {offset, size}
    const uint32_t *pool;    // adjacency entries
    uint32_t V;
    uint32_t R;
    unsigned long long pool_cap;  // entries in `pool`
};

// First index in the sorted entry list whose neighbour id is >= w (entries are (id<<1)|flag).
__device__ __forceinline__ uint32_t lower_bound_entry(const uint32_t *list, uint32_t size, uint32_t w) {
    const uint32_t key = w << 1;
    uint32_t lo = 0, hi = size;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(list + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Looks up neighbour w; returns the entry, or 0xFFFFFFFF when absent.
__device__ __forceinline__ uint32_t find_entry(const uint32_t *list, uint32_t size, uint32_t w) {
    uint32_t i = lower_bound_entry(list, size, w);
    if (i < size) {
        uint32_t e = __ldg(list + i);
        if ((e >> 1) == w) return e;
    }
    return 0xFFFFFFFFu;
}

__device__ __forceinline__ bool test_bit(const uint32_t *bits, uint32_t v) {
    return (__ldg(bits + (v >> 5)) >> (v & 31)) & 1u;
}

// Position of the first sorted batch key whose (rel, src) is >= (rel, x).
__device__ __forceinline__ uint32_t find_list_head(const unsigned long long *keys, uint32_t m, KeyLayout kl,
                                                   unsigned long long lk) {
    uint32_t lo = 0, hi = m;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (kl.list_of(__ldg(keys + mid)) < lk) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct EnumParams {
    const DevPlan *plans;
    uint32_t nplans;
    const DevTailTerm *terms;
    GraphView g;
    const uint32_t *bits;            // NLF candidate bitmaps
    uint32_t words;                  // words per bitmap
    const unsigned long long *keys;  // sorted batch keys
    uint32_t m;
    KeyLayout kl;
    const uint8_t *eff;              // CSM_EFF_* per key
    const uint32_t *seg_flagged;     // per list head: flagged entries in this phase
    uint32_t phase;
    const uint32_t *seed_lo;         // per plan: first key of its seed relation
    const uint32_t *ticket_prefix;   // per plan: prefix of seed chunks (nplans + 1)
    const WorkItem *frontier;        // alternative work source (semi-BFS frontier)
    uint32_t nfrontier;
    WorkItem *queue;                 // donation ring (qmask + 1 slots)
    unsigned long long *seq;         // per slot: epoch << 32 | position (see EnumControl)
    uint32_t qmask;
    EnumControl *ctrl;
    unsigned long long *counts;      // per plan
    uint32_t mode;                   // 0 count, 1 materialize, 2 expand one level
    uint32_t *rows;                  // materialize: rows of 1 + CSM_MAXQV words
    unsigned long long row_cap;
    WorkItem *expand_out;
    unsigned long long expand_cap;
    uint32_t donate;
    uint32_t steal_min;
    uint32_t idle_limit;             // polls of an idle warp waiting for donated work
    unsigned long long time_limit_ns;  // >0: warps stop once the launch has run this long
    const unsigned int *abort_flag;  // nonzero: the batch update failed, skip enumeration
    const uint32_t *touched;         // bit per vertex: some batch key has it as list owner
    // 1: some plan ends in a last level without a Cartesian tail, so the kernel variant with the
    // register-resident last-level loop is launched (the other variant leaves that code out,
    // which keeps the registers of the tail-counting paths).
    uint32_t last_loop;
    // Pendant counting levels (DevPlan.memo_slot): per table, the count below a prefix for every
    // data vertex at the plan's memo_depth; nullptr counts those levels like any other.
    const unsigned long long *memo;
};

#define CSM_ROW_WORDS (1 + CSM_MAXQV)
#define CSM_ENUM_MODE_COUNT 0
#define CSM_ENUM_MODE_ROWS 1
#define CSM_ENUM_MODE_EXPAND 2

size_t enum_smem_bytes(int warps_per_block);
// Resident blocks per SM of the enumeration kernel compiled for `occupancy` (4, 5 or 6)
// resident 256-thread blocks per SM.
int enum_blocks_per_sm(int warps_per_block, int occupancy);
void launch_enumerate(const EnumParams &p, int blocks, int warps_per_block, int occupancy, cudaStream_t s);
void launch_seed_tickets(const DevPlan *plans, uint32_t nplans, const unsigned long long *keys, uint32_t m,
                         KeyLayout kl, uint32_t *seed_lo, uint32_t *ticket_prefix, EnumControl *ctrl,
                         cudaStream_t s);
void launch_ctrl_reset(EnumControl *ctrl, uint32_t active, unsigned long long nticket, cudaStream_t s);
// Fills table `out` (one entry per data vertex) for the pendant plan `plan` in this phase.
void launch_pendant_counts(const EnumParams &p, uint32_t plan, unsigned long long *out, cudaStream_t s);
void launch_expand_bound(const EnumParams &p, const WorkItem *items, const unsigned long long *nitems,
                         cudaStream_t s);

}  // namespace csm
