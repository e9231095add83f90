// Matching-order planner.
//
// One plan per (query, updated query edge i).  The vertex-selection rules follow the
// reference's PlanManager (graph/plan.cpp): the BFS indexing order (plan.cpp:1548-1602),
// the GAMMA order (plan.cpp:1843-2116), the GCSM v2 order (plan.cpp:386-782) and the RI order
// (plan.cpp:195-385), with backward neighbours sorted by the average degree of their relation
// (plan.cpp:471-486).  Every order here starts with the endpoints of the updated edge, so that
// every partial embedding grows from a batch edge; where the reference's GCSM and RI rules
// pick another start, their vertex priority is kept and re-anchored at the updated edge.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "common.h"
#include "query.h"

namespace csm {

enum class Order { kIndexing = 0, kGamma = 1, kGcsm = 2, kRi = 3 };

struct PlanOptions {
    Order order = Order::kGcsm;
    bool cartesian = true;
    bool materialize = false;
};

// Summary of the candidate index per directed query edge (GetSummary, match_gpu.cu:589-609):
// card[u*nv+uu] = number of candidate edges, avg[u*nv+uu] = card / number of sources.
struct EdgeStats {
    std::vector<uint32_t> card;
    std::vector<float> avg;
};

struct HostPlan {
    std::vector<uint8_t> order;                 // query vertices by depth
    std::vector<std::vector<uint8_t>> bn;       // per depth: depths of backward neighbours
    int tail_start = 0;
    std::vector<DevTailTerm> terms;             // tail polynomial
    DevPlan dev;                                // packed form (term_begin set by the engine)
};

using RelOf = std::function<uint16_t(uint32_t u, uint32_t uu)>;  // relation of query edge u->uu

// Builds the plans of every query edge of `q`, in qe_list_ order.
std::vector<HostPlan> build_plans(const Query &q, uint16_t query_id, uint32_t nlf_base,
                                  const EdgeStats &st, const PlanOptions &opt, const RelOf &rel_of);

// Text description, one block per query edge, in the spirit of PlanManager::PrintOrders.
std::string describe_plans(const Query &q, const std::vector<HostPlan> &plans);

// Exposed for tests: the bare vertex orders.
std::vector<uint8_t> indexing_order(const Query &q, uint32_t u0, uint32_t u1);

}  // namespace csm
