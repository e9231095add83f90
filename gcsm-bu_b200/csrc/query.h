// Host-side query graph and its metadata.
//
// Mirrors the query half of the reference's GraphFileIoManager: the sorted neighbour lists
// (graph/graph.cpp:251-258), the query-edge list qe_list_ in (u, uu), u < uu order collected
// by `for u: for uu in nbrs_[u]` (graph.cpp:332-347) and the neighbour-label-frequency (NLF)
// groups (graph.cpp:295-330).  Labels stay raw here; the engine maps them to dense ids.
#pragma once

#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

namespace csm {

struct NlfGroup {
    uint32_t elabel;   // raw edge label of the group
    uint32_t vlabel;   // raw label of the neighbours in the group
    uint32_t count;    // number of query neighbours with that (edge label, vertex label)
};

struct Query {
    uint32_t nv = 0;
    uint32_t ne = 0;
    std::vector<uint32_t> vlabel;                                  // raw vertex labels
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> nbrs;  // sorted (neighbour, raw elabel)
    std::vector<std::pair<uint32_t, uint32_t>> qe_list;            // (u, uu), u < uu
    std::vector<uint32_t> qe_elabel;                               // raw label of qe_list[i]
    std::vector<int> qe_index;                                     // [u*nv+uu] -> i or -1
    std::vector<std::vector<NlfGroup>> nlf;                        // per vertex

    bool adjacent(uint32_t u, uint32_t uu) const { return qe_index[u * nv + uu] >= 0; }
    uint32_t degree(uint32_t u) const { return (uint32_t)nbrs[u].size(); }
    uint32_t edge_label(uint32_t u, uint32_t uu) const { return qe_elabel[qe_index[u * nv + uu]]; }
};

// Builds a Query from edge arrays.  Returns an empty string on success, else the reason.
std::string build_query(uint32_t nv, const uint32_t *vlabel, uint32_t ne, const uint32_t *src,
                        const uint32_t *dst, const uint32_t *elabel, Query &q);

}  // namespace csm
