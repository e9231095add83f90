// The engine behind the C ABI: owns the device graph, the candidate bitmaps, the plans and
// the per-batch scratch of one GPU.  Replaces class MatchGPU (graph/match_gpu.h:80-225) and the
// batch loop of TechniquePermutationProcess (technique_permutation.h:121-214).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/csm.h"
#include "common.h"
#include "kernels.cuh"
#include "plan.h"
#include "query.h"
#include "store.cuh"

namespace csm {

// Scratch of the enumeration kernel: control block, donation ring with its sequence words, and
// the per-plan seed ranges and ticket prefixes (3 * nplans and nplans + 1 words).
struct EnumScratch {
    EnumControl *ctrl = nullptr;
    WorkItem *queue = nullptr;
    unsigned long long *seq = nullptr;  // per-slot sequence words of the donation ring
    uint32_t qcap = 0;                  // ring slots (a power of two, >= CSM_QUEUE_MIN_SLOTS)
    uint32_t *seed_lo = nullptr;
    uint32_t *ticket_prefix = nullptr;
};

// Resources lent to the engine for one batch: enumeration scratch, two semi-BFS frontier
// buffers of frontier_cap items (a cap of 0 means depth-first search only) and the stream.
struct ExecContext {
    EnumScratch scratch;
    WorkItem *frontier[2] = {nullptr, nullptr};
    unsigned long long frontier_cap = 0;
    cudaStream_t stream = nullptr;
};

// One launch configuration of the enumeration (what the autotuner varies).
struct LaunchConfig {
    int strategy;          // search strategy 0..3
    uint32_t steal_chunk;  // smallest candidate range split by donation
    int warps_per_block;
    int occupancy;         // kernel variant: resident 256-thread blocks per SM
    uint32_t frontier_mult;  // semi-BFS stops once the frontier holds this many items per warp
};

struct Options {
    Order order = Order::kGcsm;
    int search_strategy = 2;  // 0 DFS+stealing, 1 DFS, 2 dynamic BFS-DFS, 3 BFS
    bool local_index = true;
    bool cartesian = true;
    bool heavy_vertex_avoidance = true;
    bool relation_switch = true;
};

// Resolves --algorithm presets (utils/technique_option.h:58-86).
Options resolve_options(const csm_config &cfg);

class Engine {
  public:
    explicit Engine(const csm_config &cfg);
    ~Engine();

    csm_status init();
    csm_status load_query(uint32_t nv, const uint32_t *vlabel, uint32_t ne, const uint32_t *src, const uint32_t *dst,
                          const uint32_t *elabel, int32_t *qid);
    csm_status load_graph(uint32_t nv, const uint32_t *vlabel, uint64_t ne, const uint32_t *src, const uint32_t *dst,
                          const uint32_t *elabel);
    // Device-state checkpoint of the data graph (lists with their slack); load_snapshot replaces
    // load_graph in an engine with the same registered queries.
    csm_status save_snapshot(const char *path);
    csm_status load_snapshot(const char *path);
    csm_status apply_host(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                          const uint8_t *is_delete, csm_batch_result *out);
    csm_status apply_device(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                            const uint8_t *is_delete, cudaStream_t stream, csm_batch_result *out);
    // The batch pipeline with caller-provided enumeration scratch and no allocation: batches
    // beyond the preallocated capacity are rejected and the adjacency pool is never regrown.
    csm_status apply_device_noalloc(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                                    const uint8_t *is_delete, cudaStream_t stream, const EnumScratch &scratch,
                                    csm_batch_result *out);
    // The host-array batch pipeline on borrowed scratch, frontier and stream (the serving loop
    // runs many engines on a few slots this way).
    csm_status apply_host_ctx(const ExecContext &ctx, uint64_t n, const uint32_t *src, const uint32_t *dst,
                              const uint32_t *elabel, const uint8_t *is_delete, csm_batch_result *out);
    // Largest semi-BFS frontier (items) the last batch wrote.
    unsigned long long last_frontier_rows() const { return last_frontier_rows_; }
    uint32_t num_plans() const { return (uint32_t)plans_.size(); }
    bool graph_loaded() const { return graph_loaded_; }
    // Warps of one enumeration launch (frontier estimates scale with it).
    uint64_t enum_warps() const { return (uint64_t)blocks_ * (uint64_t)warps_per_block_; }
    // Search strategy of the launch configuration in use (0..3).
    int strategy() const { return lc_.strategy; }
    // Frontier items at which the dynamic semi-BFS stops expanding.
    uint64_t semi_bfs_target_items() const { return (uint64_t)lc_.frontier_mult * enum_warps(); }
    uint64_t batch_capacity() const { return batch_cap_; }
    // Device address of the library's static scratch array for this engine, looked up with
    // `lookup` on the first call (the engine's device current).  Kept per engine: an engine
    // lives in one device context, while a context re-created after cudaDeviceReset may place
    // the array elsewhere.
    cudaError_t static_scratch(cudaError_t (*lookup)(void **), void **out) {
        if (!static_scratch_) {
            void *p = nullptr;
            const cudaError_t rc = lookup(&p);
            if (rc != cudaSuccess) return rc;
            static_scratch_ = p;
        }
        *out = static_scratch_;
        return cudaSuccess;
    }
    // Enumeration time limit for later batches (microseconds per launch, 0 = none).
    void set_time_limit_us(uint64_t us) { time_limit_us_ = us; }
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    csm_status edge_counts(int32_t qid, uint64_t *pos, uint64_t *neg, uint32_t capacity, uint32_t *n_out) const;
    csm_status embeddings(int32_t qid, int32_t sign, uint32_t **rows, uint64_t *nrows);
    csm_status describe(int32_t qid, char *buf, size_t n) const;
    csm_status stats(csm_stats *out) const;
    void reset_stats();
    csm_status memory(uint64_t *free_b, uint64_t *total_b) const;

    const std::string &error() const { return err_; }
    csm_status fail(csm_status code, const std::string &msg);
    csm_status cuda_fail(cudaError_t e, const char *where);

    uint32_t num_queries() const { return (uint32_t)queries_.size(); }

  private:
    csm_status ensure_batch_capacity(uint64_t n);
    csm_status upload_snapshot(uint64_t used, uint64_t capacity, const std::vector<uint2> &meta,
                               const std::vector<uint32_t> &cap, const std::vector<uint32_t> &pool);
    // Every device allocation of the engine.  With csm_config.inject_alloc_failure = N > 0 the
    // N-th one fails as out of memory (once): fault injection for the error paths.
    cudaError_t dev_alloc_bytes(void **p, size_t bytes) {
        if (inject_left_ > 0 && --inject_left_ == 0) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
        return cudaMalloc(p, bytes ? bytes : 1);
    }
    template <typename T>
    cudaError_t dev_alloc(T **p, size_t count) {
        return dev_alloc_bytes(reinterpret_cast<void **>(p), sizeof(T) * (count ? count : 1));
    }
    int64_t inject_left_ = 0;
    csm_status run_batch(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                         const uint8_t *is_delete, bool has_delete, cudaStream_t s, csm_batch_result *out);
    csm_status enumerate_phase(uint32_t phase, uint32_t m, cudaStream_t s);
    csm_status maybe_compact(cudaStream_t s);

    csm_config cfg_;
    Options opt_;
    std::string err_;
    int device_ = 0;
    int sm_count_ = 148;
    bool graph_loaded_ = false;
    bool poisoned_ = false;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev_[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // batch, DEL enum, INS enum

    // Queries and label spaces.
    std::vector<Query> queries_;
    std::vector<uint32_t> vlab_raw_;      // sorted raw vertex labels of all queries
    std::vector<uint32_t> elab_raw_;      // sorted raw edge labels of all queries
    std::vector<uint32_t> rel_triples_;   // rel -> (a << 16 | l << 8 | b)
    std::vector<uint16_t> rel_table_;     // host copy of the device table
    std::vector<uint32_t> nlf_base_;      // first bitmap of each query

    // Device tables.
    uint32_t *d_elab_raw_ = nullptr;
    uint16_t *d_rel_table_ = nullptr;
    uint32_t *d_spec_begin_ = nullptr;
    NlfSpec *d_specs_ = nullptr;
    uint32_t *d_bits_ = nullptr;
    uint32_t nbitmaps_ = 0;
    uint32_t words_ = 0;
    DeviceGraph g_;
    KeyLayout kl_{};

    // Plans.
    std::vector<HostPlan> plans_;
    std::vector<uint32_t> plan_begin_;    // per query, first plan (plus one past the end)
    DevPlan *d_plans_ = nullptr;
    DevTailTerm *d_terms_ = nullptr;

    // Batch buffers.
    uint64_t batch_cap_ = 0;              // updates
    uint32_t *d_upd_src_ = nullptr, *d_upd_dst_ = nullptr, *d_upd_lab_ = nullptr;
    uint8_t *d_upd_del_ = nullptr;
    uint32_t *h_pin_ = nullptr;           // pinned staging: src, dst, lab (3 * cap) + del bytes
    unsigned long long *d_keys_raw_ = nullptr, *d_keys_ = nullptr;
    void *d_sort_temp_ = nullptr;
    size_t sort_temp_bytes_ = 0;
    BatchScratch bs_;

    // Enumeration state.
    EnumControl *d_ctrl_ = nullptr;
    WorkItem *d_queue_ = nullptr;
    unsigned long long *d_seq_ = nullptr;
    uint32_t qcap_ = 0;
    uint64_t time_limit_us_ = 0;              // per enumeration launch; 0 = none
    csm_status deferred_ = CSM_OK;            // timeout / overflow of this batch, reported at its end
    bool last_loop_ = false;                  // launch the kernel variant with the last-level loop
    // Pendant plans (DevPlan.memo_slot): table t is filled each phase by the kernel of plan
    // memo_plan_[t] and read by every plan with the same counting level and tail; d_memo_ holds
    // memo_cap_ tables of V entries.
    unsigned long long *d_memo_ = nullptr;
    size_t memo_cap_ = 0;
    std::vector<uint32_t> memo_plan_;
    unsigned long long last_frontier_rows_ = 0;
    // CUDA graphs of whole batches (depth-first strategies), keyed by what the capture bakes in.
    struct GraphKey {
        uint64_t n;
        bool del;
        uint64_t gen;
        int strategy;
        uint32_t steal;
        int wpb, occ, blocks;
        bool operator==(const GraphKey &o) const {
            return n == o.n && del == o.del && gen == o.gen && strategy == o.strategy && steal == o.steal &&
                   wpb == o.wpb && occ == o.occ && blocks == o.blocks;
        }
    };
    struct GraphEntry {
        GraphKey key{};
        cudaGraphExec_t exec = nullptr;
        uint64_t kernels = 0, enum_launches = 0;
    };
    struct Stats0 {
        uint64_t kernels, enum_launches;
    };
    std::vector<GraphEntry> graphs_;
    bool capturing_ = false;
    // Timing events inside a captured graph must be event-record nodes (external events);
    // outside a capture they are ordinary records.
    cudaError_t record_event(cudaEvent_t e, cudaStream_t s) const {
        return cudaEventRecordWithFlags(e, s, capturing_ ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
    uint64_t graph_gen_ = 0;  // bumped whenever a buffer a graph refers to is reallocated
    bool graphs_on() const {
        return cfg_.cuda_graphs && !no_alloc_ && lc_.strategy < 2 && cfg_.materialize_rows == 0;
    }
    csm_status enqueue_batch(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                             const uint8_t *is_delete, bool has_delete, bool tuning, cudaStream_t s);
    csm_status enqueue_readback(cudaStream_t s);
    // Live re-planning: planner statistics, plan upload, and the drift check after a batch.
    csm_status prepare_tables(uint32_t nv, const uint32_t *vlabel, const uint8_t *vlab_dense);
    csm_status build_lists(uint64_t ne, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel, uint32_t nvl,
                           uint32_t nel);
    csm_status finish_load();
    uint64_t query_fingerprint() const;
    bool tables_ready_ = false;
    csm_status compute_edge_stats(std::vector<EdgeStats> &stats);
    csm_status install_plans(const std::vector<EdgeStats> &stats);
    csm_status maybe_replan();
    size_t terms_cap_ = 0;
    long long *d_rel_delta_ = nullptr;      // [R] net entry change of the current batch
    uint32_t *d_touched_ = nullptr;         // [words_] list owners among the batch keys
    long long *h_rel_delta_ = nullptr;      // pinned copy
    std::vector<long long> rel_size_, rel_size_planned_;
    csm_status launch_graph(uint64_t n, bool has_delete, cudaStream_t s);
    void clear_graphs();
    csm_status apply_host_on(cudaStream_t s, uint64_t n, const uint32_t *src, const uint32_t *dst,
                             const uint32_t *elabel, const uint8_t *is_delete, csm_batch_result *out);
    uint32_t *d_seed_lo_ = nullptr;       // 3 * nplans
    uint32_t *d_ticket_prefix_ = nullptr; // nplans + 1
    unsigned long long *d_counts_ = nullptr;  // per plan, per phase (2 * nplans)
    WorkItem *d_frontier_[2] = {nullptr, nullptr};
    unsigned long long frontier_cap_ = 0;
    uint32_t *d_rows_ = nullptr;
    unsigned long long row_cap_ = 0;
    unsigned long long *h_counts_ = nullptr;  // pinned readback
    EnumControl *h_ctrl_ = nullptr;           // pinned: control block of the DEL and INS launches
    unsigned long long *d_misc_ = nullptr;    // small device scratch
    bool phase_ran_[2] = {false, false};
    EnumScratch sc_;                          // scratch used by enumerate_phase
    bool no_alloc_ = false;                   // inside apply_device_noalloc
    void *static_scratch_ = nullptr;          // see static_scratch()
    int warps_per_block_ = 8;
    int occupancy_ = 4;                       // enumeration kernel variant (blocks per SM)
    int blocks_ = 0;
    LaunchConfig lc_{};                       // configuration in use
    std::vector<LaunchConfig> tune_cands_;    // autotuner candidates
    std::vector<double> tune_ms_;             // accumulated enumeration time per candidate
    int tune_left_ = 0;                       // batches still to tune on
    bool tuned_this_batch_ = false;
    cudaEvent_t tune_ev_[32] = {};
    void set_launch_config(const LaunchConfig &c);

    // Results of the last batch.
    std::vector<uint64_t> last_counts_;   // 2 * nplans
    std::vector<std::vector<uint32_t>> last_rows_[2];  // per phase, per query: flattened rows
    bool rows_valid_ = false;

    csm_stats stats_{};
};

}  // namespace csm
