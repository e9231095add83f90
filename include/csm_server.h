/*
 * csm_server.h — continuous-batching serving loop over csm engines on one GPU.
 *
 * The reference has no serving layer: its only driver is the synchronous batch loop of
 * TechniquePermutationProcess (technique_permutation.h:121-214), one query, one stream of
 * batches, one process.  This interface adds what a long-running service needs on top of the
 * engine API of csm.h, with the per-batch arithmetic unchanged:
 *
 *  - Tenants.  Each tenant is an engine (csm_create + csm_load_query + csm_load_graph) whose
 *    data graph, candidate bitmaps and per-query state stay resident on the GPU.  Once added,
 *    the engine is driven by the server only; destroy the server before the engines.
 *  - Requests.  A request is one update batch for one tenant, or for every tenant (tenant -1,
 *    e.g. replicas of one graph holding different standing queries).  csm_server_submit copies
 *    the host arrays and returns at once.  Batches of a tenant are applied in submission order.
 *  - Slots.  A fixed number of slots (CUDA streams with their own enumeration scratch) run
 *    work units, a unit being one request on one tenant.  A unit is admitted when a slot is
 *    free, its tenant has no unit in flight, and its semi-BFS frontier estimate fits the
 *    memory budget.  Units of different tenants overlap on the device.
 *  - Memory admission.  Frontier memory comes from one device arena of memory_budget bytes.
 *    A unit asks for an estimate from its tenant's recent frontiers; it gets the estimate, or
 *    less when the arena is short (the semi-BFS then stops earlier and continues depth first),
 *    and waits only while other units hold memory and less than min_frontier_bytes is free.
 *    A unit never overflows its frontier: a level that would not fit is not started.
 *
 * Counts are exact integers and do not depend on the mix: every result equals what the same
 * engine returns for the same batch sequence through csm_apply_batch.
 */
#ifndef CSM_B200_CSM_SERVER_H
#define CSM_B200_CSM_SERVER_H

#include "csm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct csm_server csm_server;

typedef struct csm_server_config {
    int32_t device;               /* CUDA device of every tenant engine */
    int32_t slots;                /* concurrent work units (streams); 0 = 4 */
    uint64_t memory_budget;       /* device bytes for the frontiers of admitted units; 0 = 8 GiB */
    uint64_t min_frontier_bytes;  /* a grant below this waits for memory (or runs depth first
                                     when nothing else is in flight); 0 = 16 MiB */
    uint32_t max_pending;         /* submit fails with CSM_ERR_LIMIT beyond this many requests
                                     not yet waited for; 0 = 4096 */
    int32_t reserved[7];
} csm_server_config;

typedef struct csm_request_info {
    int32_t status;           /* csm_status of the request: the first failing unit's code */
    uint32_t nresults;        /* per-query results of the request (tenant order, query order) */
    uint64_t arrival_ns;      /* steady clock at submit */
    uint64_t start_ns;        /* first unit admitted to a slot */
    uint64_t done_ns;         /* last unit finished, its counts on the host */
    uint64_t frontier_bytes;  /* smallest frontier grant among its units (0: depth first) */
    uint64_t device_ns;       /* sum over units of the engine's batch latency (first H2D to counts) */
    uint64_t reserved[2];
} csm_request_info;

typedef struct csm_server_stats {
    uint64_t requests;          /* requests completed */
    uint64_t units;             /* work units run */
    uint64_t units_depth_first; /* units granted no frontier memory */
    uint64_t units_shrunk;      /* units granted less than their estimate */
    uint64_t memory_waits;      /* times the oldest unit waited for frontier memory */
    uint64_t peak_frontier_bytes;  /* most frontier memory granted at one time */
    uint64_t peak_inflight;     /* most units in flight at one time */
    uint64_t reserved[5];
} csm_server_stats;

csm_status csm_server_default_config(csm_server_config *cfg);

/* Creates the server and its slots (streams, enumeration scratch, the frontier arena). */
csm_status csm_server_create(csm_server **out, const csm_server_config *cfg);

/* Adds a loaded engine on the server's device; the server drives it from now on. */
csm_status csm_server_add_tenant(csm_server *srv, csm_engine *engine, int32_t *tenant_out);

/* Queues one update batch (host arrays, copied) for `tenant`, or for every tenant when -1.
 * Same array conventions as csm_apply_batch; is_delete may be NULL. */
csm_status csm_server_submit(csm_server *srv, int32_t tenant, uint64_t n, const uint32_t *src, const uint32_t *dst,
                             const uint32_t *elabel, const uint8_t *is_delete, uint64_t *request_out);

/* Waits up to timeout_ms (negative: no limit) for a request; on completion copies up to
 * `capacity` per-query results and the request's timing, and forgets the request.  Returns
 * CSM_ERR_TIMEOUT if it is still running (call again), else the request's status. */
csm_status csm_server_wait(csm_server *srv, uint64_t request, int64_t timeout_ms, csm_request_info *info,
                           csm_batch_result *results, uint32_t capacity);

csm_status csm_server_get_stats(const csm_server *srv, csm_server_stats *out);

/* Finishes every queued request, then stops the slots and frees the server's memory (the
 * tenant engines stay alive and usable again through csm_apply_batch). */
csm_status csm_server_destroy(csm_server *srv);

/* Last error message of the server (or of the last failed csm_server_create when NULL). */
csm_status csm_server_last_error(const csm_server *srv, char *buf, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* CSM_B200_CSM_SERVER_H */
