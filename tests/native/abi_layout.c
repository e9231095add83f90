/* Prints the byte offset of every field of the C-ABI structs, one "struct.field offset" per
 * line, for comparison with the Python binding's ctypes layouts. */
#include <stddef.h>
#include <stdio.h>

#include "csm_server.h"

#define F(s, f) printf(#s "." #f " %zu\n", offsetof(s, f))

int main(void) {
    F(csm_config, device); F(csm_config, algorithm); F(csm_config, matching_order);
    F(csm_config, search_strategy); F(csm_config, local_index); F(csm_config, cartesian_product);
    F(csm_config, heavy_vertex_avoidance); F(csm_config, relation_switch); F(csm_config, pool_entries);
    F(csm_config, max_batch); F(csm_config, frontier_bytes); F(csm_config, materialize_rows);
    F(csm_config, blocks_per_sm); F(csm_config, warps_per_block); F(csm_config, steal_chunk);
    F(csm_config, occupancy); F(csm_config, autotune_batches); F(csm_config, cuda_graphs);
    F(csm_config, replan_drift_pct); F(csm_config, semi_bfs_items_per_warp);
    F(csm_config, queue_slots); F(csm_config, inject_alloc_failure); F(csm_config, time_limit_us);
    F(csm_batch_result, positive); F(csm_batch_result, negative); F(csm_batch_result, inserted);
    F(csm_batch_result, deleted); F(csm_batch_result, latency_ns); F(csm_batch_result, apply_ns);
    F(csm_batch_result, enum_ns);
    F(csm_stats, batches); F(csm_stats, enum_launches); F(csm_stats, kernel_launches);
    F(csm_stats, enum_scan_entries); F(csm_stats, enum_probes); F(csm_stats, enum_tail_lists);
    F(csm_stats, donations); F(csm_stats, enum_ns); F(csm_stats, apply_ns); F(csm_stats, pool_used);
    F(csm_stats, pool_capacity); F(csm_stats, compactions); F(csm_stats, tuned_strategy);
    F(csm_stats, tuned_steal_chunk); F(csm_stats, tuned_warps_per_block); F(csm_stats, tuned_occupancy);
    F(csm_stats, graph_launches); F(csm_stats, replans); F(csm_stats, donations_refused);
    F(csm_server_config, device); F(csm_server_config, slots); F(csm_server_config, memory_budget);
    F(csm_server_config, min_frontier_bytes); F(csm_server_config, max_pending);
    F(csm_request_info, status); F(csm_request_info, nresults); F(csm_request_info, arrival_ns);
    F(csm_request_info, start_ns); F(csm_request_info, done_ns); F(csm_request_info, frontier_bytes);
    F(csm_request_info, device_ns);
    F(csm_server_stats, requests); F(csm_server_stats, units); F(csm_server_stats, units_depth_first);
    F(csm_server_stats, units_shrunk); F(csm_server_stats, memory_waits);
    F(csm_server_stats, peak_frontier_bytes); F(csm_server_stats, peak_inflight);
    printf("sizeof.csm_config %zu\nsizeof.csm_batch_result %zu\nsizeof.csm_stats %zu\n", sizeof(csm_config),
           sizeof(csm_batch_result), sizeof(csm_stats));
    printf("sizeof.csm_server_config %zu\nsizeof.csm_request_info %zu\nsizeof.csm_server_stats %zu\n",
           sizeof(csm_server_config), sizeof(csm_request_info), sizeof(csm_server_stats));
    return 0;
}
