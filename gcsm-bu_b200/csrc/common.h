// Shared host/device definitions of the B200 continuous subgraph matching engine.
//
// Device graph layout (replaces CSR_GPU / RelationsGPU of graph/match_gpu.h:20-47):
//  - A *relation* is a directed label triple (src vertex label, edge label, dst vertex label)
//    that occurs as the orientation of some query edge.  The reference keeps one relation per
//    directed query edge (edge_idx, graph/graph.cpp:438-459); here query edges with the same
//    triple share one relation, and the per-query-edge differences (which updated edges an
//    edge may use) are expressed by a flag on each adjacency entry instead of by copies.
//  - meta[rel * V + v] = {offset, size} of v's sorted adjacency list inside `pool`;
//    cap[rel * V + v] = its slack capacity (power of two, at least 8, as indexing.cu:46-59).
//  - An adjacency entry is (neighbour << 1) | flag.  flag = 1 marks an edge that is part of
//    the batch being processed (inserted in the insertion phase, about to be deleted in the
//    deletion phase).  Sorting by entry sorts by neighbour id.
#pragma once

#include <stdint.h>

#define CSM_MAXQV 16
#define CSM_MAXQE 42
#define CSM_MAXBN 15
#define CSM_WARP 32
#define CSM_NO_REL 0xFFFFu
#define CSM_NO_LABEL 0xFFu
#define CSM_INVALID_KEY 0xFFFFFFFFFFFFFFFFull

// Effect of one sorted batch key after classification.
#define CSM_EFF_NONE 0
#define CSM_EFF_INS 1
#define CSM_EFF_DEL 2

// Phase of an enumeration launch; equals the CSM_EFF_* value its seeds carry.
#define CSM_PHASE_INS 1
#define CSM_PHASE_DEL 2

// Maximum tail-leaf bookkeeping of one plan (Cartesian flattening, kernels/cartesian_product.cu).
#define CSM_TAIL_MAXKEYS 8
#define CSM_TAIL_MAXMASKS 32
#define CSM_TAIL_MAXCLASSES 8

// One matching-order level (one query vertex) of a plan.
struct DevLevel {
    uint16_t bn_rel[CSM_MAXBN];   // relation of (backward neighbour -> this vertex)
    uint8_t bn_depth[CSM_MAXBN];  // depth of each backward neighbour in the order
    uint8_t nbn;                  // number of backward neighbours
    uint16_t old_mask;            // bit k: backward edge k must not be a batch edge
    uint8_t qv;                   // query vertex id
    uint8_t bn_base;              // first slot of this level's lists in a flat per-plan array
    // Candidate bitmap (NLF filter) of this query vertex, or CSM_NO_BITMAP when every query
    // neighbour of the vertex is a backward neighbour: a candidate adjacent to all of them
    // already has the neighbour counts the filter asks for.
    uint32_t nlf_bitmap;
    // Bit j: the query vertex at depth j < this level has this level's label.  Lists are
    // label-partitioned, so a candidate can only coincide with those prefix vertices.
    uint16_t excl_mask;
    uint16_t pad0;
    uint32_t pad1;
};

#define CSM_NO_BITMAP 0xFFFFFFFFu

struct DevTailTerm {
    int64_t coef;
    uint8_t nf;                    // number of factors
    uint8_t f[7];                  // mask ids
};

// Cartesian tail of a plan: query vertices at depth >= tail_start are leaves whose only
// neighbour is matched earlier (plan.cpp:1785-1841 TreeCartesianProduct).  Their number of
// injective assignments is counted by inclusion-exclusion over the leaves of one label.
struct DevTail {
    uint8_t nkeys;                              // distinct (parent depth, relation, old) lists
    uint8_t key_parent[CSM_TAIL_MAXKEYS];
    uint8_t key_old[CSM_TAIL_MAXKEYS];
    uint16_t key_rel[CSM_TAIL_MAXKEYS];
    // Per key, bit j set when the query vertex at depth j has the key's leaf label: only the
    // data vertices matched at those depths can sit in the key's list (labels partition the
    // relations), so injectivity exclusions search for those alone.
    uint16_t key_excl[CSM_TAIL_MAXKEYS];
    uint8_t nmasks;                             // key subsets whose intersection size is used
    uint8_t nclasses;
    uint8_t lane_par;                           // every mask is one key: count 32 prefixes per warp step
    uint16_t mask[CSM_TAIL_MAXMASKS];
    uint16_t class_term_begin[CSM_TAIL_MAXCLASSES + 1];  // into the plan's term list
};

// One (query, updated query edge) pair: the unit of the per-batch decomposition of
// technique_permutation.h:125-212.
struct DevPlan {
    uint16_t query;
    uint8_t n;             // number of query vertices
    uint8_t qe;            // index of the updated query edge in qe_list_
    uint8_t tail_start;    // first depth of the Cartesian tail (== n when there is none)
    uint8_t materialize;   // 1: write full rows instead of counting the tail
    uint16_t seed_rel;     // relation of (order[0] -> order[1])
    uint8_t order[CSM_MAXQV];
    uint32_t nlf0, nlf1;   // candidate bitmaps of order[0] and order[1]
    uint32_t term_begin;   // tail polynomial terms in the global term array
    uint32_t nterms;
    DevLevel lv[CSM_MAXQV];
    DevTail tail;
    // 1 when there is no tail and the last query vertex has no backward neighbour at depth
    // n - 2: its candidates then depend only on the prefix f[0..n-3], so they are counted once
    // per such prefix, and each vertex at depth n - 2 subtracts one when it is itself one of
    // them (injectivity; possible only when the two query vertices share a label).
    uint8_t shared_last;
    // Items of this depth or deeper pass a breadth-first expansion unexpanded: tail_start - 1,
    // n - 2 for shared_last plans (whose level n - 2 stays whole inside one item), tail_start - 2
    // for pendant plans (whose counting level is never entered).
    uint8_t expand_stop;
    // Pendant counting level: the counting level c = tail_start - 1 has one backward neighbour,
    // at depth memo_depth, every tail list hangs off c itself, and no prefix vertex shares a label
    // with c or a tail vertex.  The count below a prefix is then a function of the one data vertex
    // at memo_depth, precomputed for every vertex per phase into table memo_slot (CSM_NO_MEMO:
    // not pendant; CSM_MEMO_PENDING: pendant, no table assigned yet).
    uint8_t memo_slot;
    uint8_t memo_depth;
};

#define CSM_NO_MEMO 0xFFu
#define CSM_MEMO_PENDING 0xFEu

// Work item of the persistent enumeration: a partial embedding with `depth` fixed vertices
// and the range [lo, hi) of candidates still to scan at level `depth` (for depth 0 the range
// indexes seed positions in the sorted batch).
struct WorkItem {
    uint32_t plan;
    uint32_t depth;
    uint32_t lo;
    uint32_t hi;
    uint32_t f[CSM_MAXQV];
};

// Device-side control block of one enumeration launch.
//
// The donation queue is a ring of `qcap` (a power of two, at least 32) slots addressed by
// monotone 32-bit positions: position p lives in slot p & (qcap - 1).  Each slot carries a
// 64-bit sequence word (epoch << 32 | position): the producer of position p may write the slot
// once its word reads (epoch, p) — or, in the first lap, any older epoch — and publishes with
// (epoch, p + 1); the consumer that takes p releases the slot with (epoch, p + qcap).  Slots are
// reused for the whole launch, no position is ever skipped, and nobody waits on a slot.
struct EnumControl {
    unsigned long long ticket;        // next seed / frontier ticket
    unsigned long long nticket;       // total tickets
    unsigned int q_head;              // donation positions reserved
    unsigned int q_tail;              // donation positions claimed
    unsigned int hungry;              // outstanding work requests of idle warps
    unsigned int active;              // warps holding work
    unsigned int error;               // CSM_ERRBIT_* of this launch
    unsigned int epoch;               // launch epoch, stamps the queue's sequence words
    unsigned long long out_rows;      // rows written (materialize / expand)
    unsigned long long scan_entries;  // statistics
    unsigned long long probes;
    unsigned long long tail_lists;
    unsigned long long donations;
    unsigned long long expand_bound;  // upper bound of the next BFS level
    unsigned long long t_start;       // device clock (ns) when the launch's control block was reset
    unsigned long long queue_full;    // donations refused because the ring was full
    unsigned long long shared_last;   // last levels counted once for a prefix (DevPlan.shared_last)
    // First failed consistency check of the launch (CSM_ERRBIT_CORRUPT): where (CSM_BAD_*) and
    // three values describing it.  The offending item, list or entry is skipped, not used.
    unsigned int bad_where;
    unsigned int bad_a, bad_b, bad_c;
};

#define CSM_BAD_ITEM 1u      // a claimed work item: a = plan, b = depth, c = ring position
#define CSM_BAD_FRONTIER 2u  // a frontier item: a = plan, b = depth, c = ticket
#define CSM_BAD_LIST 3u      // a list-table entry past the pool: a = offset, b = size, c = level
#define CSM_BAD_ENTRY 4u     // an adjacency entry naming no vertex: a = entry, b = offset, c = level

// Positions past this are never reserved (a launch would need 2^31 donations to reach it).
#define CSM_QUEUE_POS_LIMIT 0x7FFFFFFFu
#define CSM_QUEUE_MIN_SLOTS 32u

#define CSM_ERRBIT_TIMEOUT 1u  // the launch ran past its time limit and stopped early
#define CSM_ERRBIT_OUTPUT 2u
#define CSM_ERRBIT_POOL 8u
#define CSM_ERRBIT_CORRUPT 16u  // a consistency check failed (see EnumControl.bad_*)
