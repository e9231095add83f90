/*
 * csm.h — C ABI of the B200 batch-update continuous subgraph matching engine (libcsm.so).
 *
 * The reference (gh8li/GCSM-BU) exposes no library: its only public boundary is the `csmg`
 * process (main.cpp:162-190) and, inside that process, class MatchGPU
 * (graph/match_gpu.h:80-225) driven by TechniquePermutationProcess
 * (technique_permutation.h:29-225).  Every entry point below replaces one step of that
 * driver; the comment on each names the reference code it stands in for.  The `csmg`
 * command-line tool shipped with this library is a thin caller of these functions.
 *
 * Conventions
 *  - Every function returns csm_status: CSM_OK (0) or a negative error code.  Nothing
 *    calls exit() or aborts; csm_last_error() gives a one-line reason.
 *  - Host arrays are owned by the caller and only read during the call.  Device state is
 *    owned by the engine.  One engine drives one GPU; calls on one engine must not run
 *    concurrently from several host threads.
 *  - Vertex ids are dense uint32 in [0, nv).  Labels are the raw uint32 values of the
 *    `v`/`e` text formats; the engine keeps only labels that occur in a registered query
 *    (graph/graph.cpp:389-433 drops the rest the same way).
 *  - Edges are undirected (graph/graph.cpp:251-258, :435-459).  A batch is the set
 *    operation G' = (G \ deletions) U insertions; self-loops and repeated lines are ignored.
 */
#ifndef CSM_B200_CSM_H
#define CSM_B200_CSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t csm_status;

#define CSM_OK 0
#define CSM_ERR_INVALID_ARG (-1)
#define CSM_ERR_CUDA (-2)
#define CSM_ERR_OOM (-3)
#define CSM_ERR_TIMEOUT (-4)
#define CSM_ERR_STATE (-5)
#define CSM_ERR_LIMIT (-6)
#define CSM_ERR_OVERFLOW (-7)
#define CSM_ERR_NO_DEVICE (-8)

/* Query size limits, as utils/config.h:9-10 of the reference. */
#define CSM_MAX_QV 16
#define CSM_MAX_QE 42

typedef struct csm_engine csm_engine;

/*
 * Engine configuration.  `algorithm` and the ablation switches carry the meaning of the
 * reference's --algorithm / --matching_order / --search_strategy / --local_index /
 * --cartesian_product / --heavy_vertex_avoidance / --relation_switch flags
 * (utils/technique_option.h:58-86).  A value of -1 for a switch means "the preset of
 * `algorithm`" (presets at utils/technique_option.h:60-71).
 */
typedef struct csm_config {
    int32_t device;                 /* CUDA device ordinal (main.cpp:179) */
    int32_t algorithm;              /* 0..5; 0 reads the switches below */
    int32_t matching_order;         /* 0 indexing(BFS), 1 GAMMA, 2 GCSM, 3 RI */
    int32_t search_strategy;        /* 0 DFS+stealing, 1 DFS, 2 dynamic BFS-DFS, 3 BFS */
    int32_t local_index;            /* 0/1 */
    int32_t cartesian_product;      /* 0/1 */
    int32_t heavy_vertex_avoidance; /* 0/1 (accepted; no effect on counts) */
    int32_t relation_switch;        /* 0/1 (accepted; no effect on counts) */
    uint64_t pool_entries;          /* adjacency pool size in uint32 entries; 0 = automatic */
    uint64_t max_batch;             /* largest batch (update lines) to preallocate for; 0 = 1<<20 */
    uint64_t frontier_bytes;        /* semi-BFS frontier budget in bytes; 0 = automatic */
    uint64_t materialize_rows;      /* >0: keep up to this many embedding rows per batch */
    int32_t blocks_per_sm;          /* persistent enumeration launch shape; 0 = automatic */
    int32_t warps_per_block;        /* 0 = automatic */
    int32_t steal_chunk;            /* minimum candidate range split by work donation; 0 = 8 */
    int32_t occupancy;              /* enumeration kernel built for 4, 5 or 6 resident 256-thread
                                       blocks per SM (fewer registers per thread); 0 = 4 */
    int32_t autotune_batches;       /* >0: over the first batches, time the enumeration under every
                                       candidate launch configuration and keep the fastest */
    int32_t cuda_graphs;            /* nonzero: replay each batch's device work from a CUDA graph
                                       (depth-first strategies 0 and 1; one capture per batch size) */
    int32_t replan_drift_pct;       /* >0: re-plan the matching orders after a batch that moved a
                                       relation's size by more than this percentage since the last
                                       planning (the reference plans once, before the stream) */
    int32_t semi_bfs_items_per_warp; /* dynamic semi-BFS (strategy 2) stops expanding once the
                                       frontier holds this many items per warp; 0 = 512 */
    int32_t queue_slots;            /* work-donation ring of the enumeration: slots, a power of two
                                       in [32, 2^24]; 0 = 2^18 (a full ring only costs balance) */
    int32_t inject_alloc_failure;   /* >0: the engine's N-th device allocation fails as out of memory
                                       (once); fault injection for testing callers' error paths */
    uint64_t time_limit_us;         /* >0: every enumeration launch stops after this many
                                       microseconds; see csm_set_time_limit */
} csm_config;

/* Per-query result of one batch. */
typedef struct csm_batch_result {
    uint64_t positive;   /* new embeddings (technique_permutation.h:224 "Num Positive Matches") */
    uint64_t negative;   /* embeddings destroyed by deletions (no reference counterpart) */
    uint64_t inserted;   /* effective undirected edge insertions of the batch */
    uint64_t deleted;    /* effective undirected edge deletions of the batch */
    uint64_t latency_ns; /* device time of the whole batch (same for every query of a batch) */
    uint64_t apply_ns;   /* device time spent applying updates and refreshing candidates */
    uint64_t enum_ns;    /* device time spent enumerating */
    uint64_t reserved;
} csm_batch_result;

/* Engine-wide counters, cumulative since csm_create (or csm_reset_stats). */
typedef struct csm_stats {
    uint64_t batches;
    uint64_t enum_launches;         /* persistent enumeration launches */
    uint64_t kernel_launches;       /* every kernel launch of the library */
    uint64_t enum_scan_entries;     /* adjacency entries read by candidate scans */
    uint64_t enum_probes;           /* membership probes (one sorted-list lookup each) */
    uint64_t enum_tail_lists;       /* tail-leaf lists sized arithmetically */
    uint64_t donations;             /* work items split off by work donation */
    uint64_t enum_ns;               /* device time inside enumeration launches */
    uint64_t apply_ns;              /* device time inside update/index kernels */
    uint64_t pool_used;             /* adjacency pool entries in use */
    uint64_t pool_capacity;
    uint64_t compactions;           /* pool compactions (slack re-layout) */
    uint64_t tuned_strategy;        /* launch configuration in use (chosen by the autotuner, or */
    uint64_t tuned_steal_chunk;     /* the configured one) */
    uint64_t tuned_warps_per_block;
    uint64_t tuned_occupancy;
    uint64_t graph_launches;        /* batches replayed from a CUDA graph */
    uint64_t replans;               /* re-plannings triggered by relation-size drift */
    uint64_t donations_refused;     /* donations not made because the donation ring was full */
    uint64_t enum_shared_last;      /* last query levels counted once for all vertices matched at
                                       the level above (the last vertex is not adjacent to it) */
} csm_stats;

/* Fills `cfg` with the defaults (algorithm 0 with all switches on, as main.cpp). */
csm_status csm_default_config(csm_config *cfg);

/* Replaces MatchGPU::MatchGPU (graph/match_gpu.cu:84-128) and cudaSetDevice (main.cpp:179). */
csm_status csm_create(csm_engine **out, const csm_config *cfg);

/* Replaces MatchGPU::~MatchGPU and DeallocOnline/DeallocRelations (match_gpu.cu:178-204, 379-405, 516-535). */
csm_status csm_destroy(csm_engine *engine);

/*
 * Registers one standing query.  Replaces the query half of GraphFileIoManager
 * (graph/graph.cpp:191-357: parse, label remap, NLF, qe_list_).  Query vertices are
 * 0..nv-1; edges are undirected, (src, dst, elabel).  Must be called before csm_load_graph.
 * The query must be connected, with 2..16 vertices and at most 42 edges.
 */
csm_status csm_load_query(csm_engine *engine, uint32_t nv, const uint32_t *vlabel, uint32_t ne,
                          const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                          int32_t *query_id_out);

/*
 * Loads the initial data graph and builds every device structure: replaces LoadInitial
 * (graph.cpp:359-468), BuildTries + AllocRelations (match_gpu.cu:302, 336-377), the offline
 * UpdateGlobalIndex pass (technique_permutation.h:80-87) and, from the resulting candidate
 * statistics (GetSummary, match_gpu.cu:589-609), the matching plans (plan.cpp:2117-2145).
 * Vertices whose label is -1 (0xFFFFFFFF) are absent.
 */
csm_status csm_load_graph(csm_engine *engine, uint32_t nv, const uint32_t *vlabel, uint64_t ne,
                          const uint32_t *src, const uint32_t *dst, const uint32_t *elabel);

/*
 * Device-state checkpoint (no counterpart in the reference, which re-reads and re-indexes its
 * text files on every start, technique_permutation.h:28-107).  csm_save_snapshot writes the
 * data graph as it stands after the last completed batch — the label-partitioned adjacency
 * lists with their slack — to a binary file.  csm_load_snapshot takes the place of
 * csm_load_graph in an engine whose registered queries are the same (checked by fingerprint);
 * candidate bitmaps and plans are rebuilt from the restored lists.
 */
csm_status csm_save_snapshot(csm_engine *engine, const char *path);
csm_status csm_load_snapshot(csm_engine *engine, const char *path);

/*
 * Applies one update batch and counts its incremental matches for every registered query.
 * Replaces one iteration of the batch loop at technique_permutation.h:127-214 (BuildTries,
 * UpdateGlobalIndex, BuildLocalIndex_v2 and Match for every query edge).  `is_delete` may be
 * NULL (insert-only, the only form the reference reads: graph.cpp:482-563).
 * `per_query_out` receives one csm_batch_result per registered query, in query-id order.
 */
csm_status csm_apply_batch(csm_engine *engine, uint64_t n, const uint32_t *src, const uint32_t *dst,
                           const uint32_t *elabel, const uint8_t *is_delete,
                           csm_batch_result *per_query_out);

/*
 * Same as csm_apply_batch, with the four update arrays already in device memory (as
 * cudaMalloc'd by the caller); `d_is_delete` may be NULL.  No host<->device copy of the
 * updates takes place.  `stream` is a cudaStream_t (NULL = the engine's own stream).
 */
csm_status csm_apply_batch_device(csm_engine *engine, uint64_t n, const uint32_t *d_src,
                                  const uint32_t *d_dst, const uint32_t *d_elabel,
                                  const uint8_t *d_is_delete, void *stream,
                                  csm_batch_result *per_query_out);

/*
 * No counterpart in the reference.  csm_apply_batch_device for callers that cannot allocate
 * device memory while they apply updates (processes that reserve their whole memory budget up
 * front, hosts that own all device memory).  The call allocates nothing: the enumeration
 * kernel's scratch lives in one array of CSM_STATIC_SCRATCH_BYTES compiled into the library,
 * which every GPU that loads the library holds until the process exits.
 *  - Limits: at most CSM_STATIC_MAX_PLANS query edges over all registered queries, and no
 *    more updates than the batch capacity preallocated when the graph was loaded
 *    (csm_config.max_batch); larger requests fail with CSM_ERR_LIMIT.  The work-donation ring
 *    in the array has 65,536 slots (a full ring only costs balance, never a result).
 *  - The adjacency pool is never compacted or regrown here.  A batch that could need more
 *    room than is free (64 entries per update plus 2^20) is refused with CSM_ERR_LIMIT before
 *    anything changes: apply a batch through csm_apply_batch_device (which compacts), or size
 *    csm_config.pool_entries for the stream.  Should the pool still run out inside a batch,
 *    the call fails with CSM_ERR_OOM and the engine refuses every later batch (recreate it).
 *  - The first call of each engine looks up the array's device address; make that first call
 *    before any stream capture.
 *  - All calls on one device share the array, which keeps the last call's contents; nothing
 *    in it needs clearing (the control block is rewritten before every launch and the ring's
 *    sequence words carry a launch epoch).  Calls that overlap on the GPU — other streams,
 *    other engines, other threads — race on it: serialise them.
 */
#define CSM_STATIC_SCRATCH_BYTES (8u << 20)
#define CSM_STATIC_MAX_PLANS 4096u
csm_status csm_apply_batch_device_static(csm_engine *engine, uint64_t n, const uint32_t *d_src,
                                         const uint32_t *d_dst, const uint32_t *d_elabel,
                                         const uint8_t *d_is_delete, void *stream,
                                         csm_batch_result *per_query_out);

/*
 * Bounds the enumeration time of later batches (no counterpart in the reference, whose
 * kernels run to completion however long that takes).  Each enumeration launch of a batch
 * stops once it has run `time_limit_us` microseconds (0 = no limit; the initial value is
 * csm_config.time_limit_us).  A batch that hits the limit is still applied to the data graph in
 * full — the update and index kernels do not depend on the counts — but its counts are
 * incomplete: the call returns CSM_ERR_TIMEOUT with the partial counts in per_query_out, and
 * the engine stays usable for the next batch.
 */
csm_status csm_set_time_limit(csm_engine *engine, uint64_t time_limit_us);

/*
 * Per-query-edge split of the last batch's counts, in the query's qe_list_ order
 * (graph.cpp:332-347): entry i counts the embeddings whose last query edge mapped to an
 * updated data edge is qe_list_[i] (the decomposition of technique_permutation.h:125-212).
 */
csm_status csm_get_edge_counts(const csm_engine *engine, int32_t query_id, uint64_t *positive,
                               uint64_t *negative, uint32_t capacity, uint32_t *n_edges_out);

/*
 * Embedding rows of the last batch (needs cfg.materialize_rows > 0).  sign = +1 for new
 * embeddings, -1 for destroyed ones.  Rows hold nv vertex ids in query-vertex order and are
 * sorted lexicographically.  *rows_out is allocated by the library; release it with csm_free.
 * The reference never materialises rows on this path (match_gpu.cu:2101-2106).
 */
csm_status csm_get_embeddings(csm_engine *engine, int32_t query_id, int32_t sign,
                              uint32_t **rows_out, uint64_t *nrows_out);

/* Releases memory returned by csm_get_embeddings. */
csm_status csm_free(void *ptr);

/* Human-readable matching plan of one query (plan.cpp:1200-1291 PrintOrders). */
csm_status csm_describe_plan(const csm_engine *engine, int32_t query_id, char *buf, size_t n);

csm_status csm_get_stats(const csm_engine *engine, csm_stats *out);
csm_status csm_reset_stats(csm_engine *engine);

/* Device memory: used and total bytes (technique_permutation.h:21-26 print_gpu_memory). */
csm_status csm_device_memory(const csm_engine *engine, uint64_t *free_bytes, uint64_t *total_bytes);

/* Copies the last error message of `engine` (or of the last failed csm_create when NULL). */
csm_status csm_last_error(const csm_engine *engine, char *buf, size_t n);

/* Library version string, e.g. "csm-b200 0.1". */
const char *csm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CSM_B200_CSM_H */
