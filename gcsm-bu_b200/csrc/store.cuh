// Device-side structures of the graph store and the host entry points of store.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "common.h"
#include "kernels.cuh"

namespace csm {

// Candidate (NLF) rule of one query vertex: v qualifies if, for every group g,
// |N_rel[g](v)| >= cnt[g] (graph.cpp:295-330, indexing.cu:303-337).
struct NlfSpec {
    uint32_t bitmap;
    uint32_t ngroups;
    uint16_t rel[CSM_MAXQV];
    uint16_t cnt[CSM_MAXQV];
};

struct NlfTables {
    const uint32_t *spec_begin;  // [nvl + 1] specs of each dense vertex label
    const NlfSpec *specs;
    uint32_t *bits;              // [nbitmaps * words]
    uint32_t words;
};

struct LabelTables {
    const uint32_t *elab_raw;    // sorted raw edge labels
    uint32_t nel;
    const uint16_t *rel_table;   // [(a * nel + l) * nvl + b] -> relation or CSM_NO_REL
    uint32_t nvl;
};

struct DeviceGraph {
    uint32_t V = 0;
    uint32_t R = 0;
    uint2 *meta = nullptr;                 // [R * V]
    uint32_t *cap = nullptr;               // [R * V]
    uint32_t *pool = nullptr;
    unsigned long long pool_cap = 0;
    unsigned long long *pool_top = nullptr;  // device bump pointer
    uint8_t *vlab = nullptr;               // [V] dense label or CSM_NO_LABEL
    GraphView view() const { return GraphView{meta, pool, V, R, pool_cap}; }
};

// Per-batch device scratch, sized for the largest batch.
struct BatchScratch {
    uint8_t *eff = nullptr;           // [m]
    uint32_t *heads = nullptr;        // [m]
    unsigned int *nheads = nullptr;   // [1]
    uint32_t *seg_nins = nullptr;     // [m], valid at heads
    uint32_t *seg_ndel = nullptr;
    uint32_t *seg_end = nullptr;
    uint32_t *scr_y = nullptr;        // [m]
    uint32_t *scr_lb = nullptr;       // [m]
    unsigned long long *counters = nullptr;  // [2] effective insertions, deletions
    unsigned int *error = nullptr;    // [1]
};

void store_build_keys(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elab, const uint8_t *isdel,
                      const LabelTables &lt, const DeviceGraph &g, KeyLayout kl, unsigned long long *keys,
                      cudaStream_t s);
cudaError_t store_sort_keys(void *temp, size_t &temp_bytes, const unsigned long long *in, unsigned long long *out,
                            uint32_t m, KeyLayout kl, cudaStream_t s);
void store_classify(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                    cudaStream_t s);
void store_delete(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                  cudaStream_t s);
void store_insert(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                  cudaStream_t s);
void store_nlf_update(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                      const NlfTables &nt, cudaStream_t s);
void store_clear_ins(uint32_t m, const unsigned long long *keys, KeyLayout kl, DeviceGraph &g, BatchScratch &b,
                     cudaStream_t s);
void store_nlf_all(DeviceGraph &g, const NlfTables &nt, cudaStream_t s);
// Per-relation net entry change of a classified batch (delta[R], accumulated).
void store_rel_delta(uint32_t m, const unsigned long long *keys, KeyLayout kl, const BatchScratch &b, long long *delta,
                     cudaStream_t s);
// Bit per vertex owning a list that a batch key belongs to (bits[words], cleared first).
void store_touched(uint32_t m, const unsigned long long *keys, KeyLayout kl, uint32_t *bits, uint32_t words,
                   cudaStream_t s);
// Per-relation entry counts (out[R], accumulated).
void store_rel_sizes(const DeviceGraph &g, unsigned long long *out, cudaStream_t s);
void store_edge_stats(DeviceGraph &g, uint32_t rel, const uint32_t *bits_u, const uint32_t *bits_uu,
                      unsigned long long *out, cudaStream_t s);
cudaError_t store_build_from_keys(DeviceGraph &g, const unsigned long long *keys_sorted, uint32_t m, KeyLayout kl,
                                  cudaStream_t s, std::string &err);
// Compaction in two steps: store_layout computes a fresh-slack layout of the current lists
// (offsets per list, allocated by the call, and the entries it needs) without changing the
// graph; store_relayout moves the lists into a new pool along it and makes it current.
cudaError_t store_layout(const DeviceGraph &g, unsigned long long **offsets, unsigned long long &total, cudaStream_t s);
cudaError_t store_relayout(DeviceGraph &g, uint32_t *new_pool, const unsigned long long *offsets,
                           unsigned long long total, cudaStream_t s);

}  // namespace csm
