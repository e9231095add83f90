// Engine orchestration: set-up, initial load, the per-batch pipeline and result readback.
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>

namespace csm {

namespace {

uint32_t bits_for(uint64_t v) {  // bits needed to represent 0..v
    uint32_t b = 1;
    while (b < 64 && (v >> b) != 0) b++;
    return b;
}

}  // namespace

// One-line description of a failed device consistency check (EnumControl.bad_*).
static std::string describe_bad(const EnumControl &c) {
    static const char *what[] = {"?", "claimed work item (plan, depth, ring position)",
                                 "frontier item (plan, depth, ticket)", "list-table entry (offset or vertex, size or relation, level)",
                                 "adjacency entry (entry, pool index, level)"};
    const uint32_t w = c.bad_where < 5 ? c.bad_where : 0;
    return std::string("device consistency check failed: ") + what[w] + " = (" + std::to_string(c.bad_a) + ", " +
           std::to_string(c.bad_b) + ", " + std::to_string(c.bad_c) + "); the batch was abandoned";
}

Options resolve_options(const csm_config &cfg) {
    Options o;
    switch (cfg.algorithm) {
        case 1:  // GCSM-BU
            o = {Order::kGcsm, 2, true, true, true, true};
            break;
        case 2:  // QO-GAMMA
            o = {Order::kGamma, 0, false, true, false, false};
            break;
        case 4:
            o = {Order::kIndexing, 2, false, true, true, true};
            break;
        case 5:
            o = {Order::kGamma, 2, false, true, true, true};
            break;
        default: {
            o.order = cfg.matching_order >= 0 && cfg.matching_order <= 3 ? (Order)cfg.matching_order : Order::kGcsm;
            o.search_strategy = cfg.search_strategy >= 0 && cfg.search_strategy <= 3 ? cfg.search_strategy : 2;
            o.local_index = cfg.local_index != 0;
            o.cartesian = cfg.cartesian_product != 0;
            o.heavy_vertex_avoidance = cfg.heavy_vertex_avoidance != 0;
            o.relation_switch = cfg.relation_switch != 0;
        }
    }
    return o;
}

Engine::Engine(const csm_config &cfg) : cfg_(cfg), opt_(resolve_options(cfg)) {}

csm_status Engine::fail(csm_status code, const std::string &msg) {
    err_ = msg;
    return code;
}

csm_status Engine::cuda_fail(cudaError_t e, const char *where) {
    err_ = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? CSM_ERR_OOM : CSM_ERR_CUDA;
}

#define CSM_CUDA(call)                                   \
    do {                                                 \
        cudaError_t e__ = (call);                        \
        if (e__ != cudaSuccess) return cuda_fail(e__, #call); \
    } while (0)

void Engine::set_launch_config(const LaunchConfig &c) {
    // Persistent launch: never more blocks than can be resident at once.  Warps that run out
    // of work wait for the others while any warp holds work, so a block that could only start
    // after resident blocks exit would stall the launch until the idle bound runs out.
    lc_ = c;
    warps_per_block_ = c.warps_per_block;
    occupancy_ = c.occupancy;
    const int resident = enum_blocks_per_sm(warps_per_block_, occupancy_);
    const int bps = cfg_.blocks_per_sm > 0 && cfg_.blocks_per_sm < resident ? cfg_.blocks_per_sm : resident;
    blocks_ = sm_count_ * bps;
    stats_.tuned_strategy = (uint64_t)c.strategy;
    stats_.tuned_steal_chunk = c.steal_chunk;
    stats_.tuned_warps_per_block = (uint64_t)c.warps_per_block;
    stats_.tuned_occupancy = (uint64_t)c.occupancy;
}

csm_status Engine::init() {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CSM_ERR_NO_DEVICE, "no CUDA device");
    if (cfg_.device < 0 || cfg_.device >= ndev) return fail(CSM_ERR_INVALID_ARG, "device ordinal out of range");
    device_ = cfg_.device;
    CSM_CUDA(cudaSetDevice(device_));
    cudaDeviceProp prop;
    CSM_CUDA(cudaGetDeviceProperties(&prop, device_));
    if (prop.major < 10) return fail(CSM_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");
    sm_count_ = prop.multiProcessorCount;
    CSM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (auto &e : ev_) CSM_CUDA(cudaEventCreate(&e));
    if (cfg_.queue_slots != 0) {
        const uint32_t q = (uint32_t)cfg_.queue_slots;
        if (cfg_.queue_slots < (int32_t)CSM_QUEUE_MIN_SLOTS || cfg_.queue_slots > (1 << 24) || (q & (q - 1)) != 0)
            return fail(CSM_ERR_INVALID_ARG, "queue_slots must be a power of two in [32, 2^24]");
        qcap_ = q;
    } else {
        qcap_ = 1u << 18;
    }
    time_limit_us_ = cfg_.time_limit_us;
    inject_left_ = cfg_.inject_alloc_failure > 0 ? cfg_.inject_alloc_failure : 0;
    warps_per_block_ = cfg_.warps_per_block > 0 && cfg_.warps_per_block <= 8 ? cfg_.warps_per_block : 8;
    LaunchConfig lc;
    lc.strategy = opt_.search_strategy;
    // Fine donation: once the counting shortcuts made a phase tens of milliseconds long, splitting
    // ranges down to 8 candidates balanced the end of each launch best (4-16 within noise).
    lc.steal_chunk = cfg_.steal_chunk > 0 ? (uint32_t)cfg_.steal_chunk : 8u;
    lc.warps_per_block = warps_per_block_;
    lc.occupancy = cfg_.occupancy >= 4 && cfg_.occupancy <= 6 ? cfg_.occupancy : 4;
    lc.frontier_mult = cfg_.semi_bfs_items_per_warp > 0 ? (uint32_t)cfg_.semi_bfs_items_per_warp : 512u;
    set_launch_config(lc);
    if (cfg_.autotune_batches > 0) {
        // Candidates: the configured one first, then variations of one knob each: the search
        // strategy (depth first with stealing, dynamic semi-BFS, BFS while the frontier fits),
        // the semi-BFS frontier target, steal granularity, warps per block and the
        // 6-blocks-per-SM kernel variant.
        tune_cands_.push_back(lc);
        auto add = [&](LaunchConfig c) {
            for (auto &o : tune_cands_)
                if (o.strategy == c.strategy && o.steal_chunk == c.steal_chunk && o.warps_per_block == c.warps_per_block &&
                    o.occupancy == c.occupancy && o.frontier_mult == c.frontier_mult)
                    return;
            tune_cands_.push_back(c);
        };
        LaunchConfig c;
        for (int st : {0, 2, 3}) {
            c = lc;
            c.strategy = st;
            add(c);
        }
        for (uint32_t fm : {8u, 64u, 512u}) {
            c = lc;
            c.strategy = 2;
            c.frontier_mult = fm;
            add(c);
        }
        c = lc;
        c.steal_chunk = 64;  // coarser donation
        add(c);
        c = lc;
        c.warps_per_block = 4;
        add(c);
        c = lc;
        c.occupancy = 6;
        add(c);
        tune_ms_.assign(tune_cands_.size(), 0.0);
        tune_left_ = cfg_.autotune_batches;
        for (size_t i = 0; i < 2 * tune_cands_.size(); i++) CSM_CUDA(cudaEventCreate(&tune_ev_[i]));
    }
    CSM_CUDA(dev_alloc(&d_ctrl_, 1));
    CSM_CUDA(cudaMemset(d_ctrl_, 0, sizeof(EnumControl)));
    CSM_CUDA(dev_alloc(&d_misc_, 8));
    CSM_CUDA(cudaMallocHost(&h_counts_, sizeof(unsigned long long) * 64));
    CSM_CUDA(cudaMallocHost(&h_ctrl_, sizeof(EnumControl) * 2));
    return CSM_OK;
}

Engine::~Engine() {
    if (stream_) cudaStreamSynchronize(stream_);
    clear_graphs();
    void *dev[] = {d_elab_raw_, d_rel_table_, d_spec_begin_, d_specs_, d_bits_, g_.meta, g_.cap, g_.pool, g_.pool_top,
                   g_.vlab, d_plans_, d_terms_, d_upd_src_, d_upd_dst_, d_upd_lab_, d_upd_del_, d_keys_raw_, d_keys_,
                   d_sort_temp_, bs_.eff, bs_.heads, bs_.nheads, bs_.seg_nins, bs_.seg_ndel, bs_.seg_end, bs_.scr_y,
                   bs_.scr_lb, bs_.counters, bs_.error, d_ctrl_, d_queue_, d_seq_, d_seed_lo_, d_ticket_prefix_,
                   d_counts_, d_frontier_[0], d_frontier_[1], d_rows_, d_misc_, d_rel_delta_, d_touched_, d_memo_};
    for (void *p : dev)
        if (p) cudaFree(p);
    if (h_pin_) cudaFreeHost(h_pin_);
    if (h_counts_) cudaFreeHost(h_counts_);
    if (h_ctrl_) cudaFreeHost(h_ctrl_);
    for (auto &e : ev_)
        if (e) cudaEventDestroy(e);
    for (auto &e : tune_ev_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

csm_status Engine::load_query(uint32_t nv, const uint32_t *vlabel, uint32_t ne, const uint32_t *src,
                              const uint32_t *dst, const uint32_t *elabel, int32_t *qid) {
    if (graph_loaded_) return fail(CSM_ERR_STATE, "queries must be registered before the data graph is loaded");
    if (!vlabel || !src || !dst || !elabel) return fail(CSM_ERR_INVALID_ARG, "null query array");
    Query q;
    std::string why = build_query(nv, vlabel, ne, src, dst, elabel, q);
    if (!why.empty()) return fail(CSM_ERR_LIMIT, why);
    if (queries_.size() >= 4096) return fail(CSM_ERR_LIMIT, "too many standing queries");
    queries_.push_back(std::move(q));
    if (qid) *qid = (int32_t)queries_.size() - 1;
    return CSM_OK;
}

csm_status Engine::load_graph(uint32_t nv, const uint32_t *vlabel, uint64_t ne, const uint32_t *src,
                              const uint32_t *dst, const uint32_t *elabel) {
    if (graph_loaded_ || tables_ready_) return fail(CSM_ERR_STATE, "the data graph is already loaded");
    if (queries_.empty()) return fail(CSM_ERR_STATE, "register at least one query before loading the graph");
    if (nv == 0 || !vlabel) return fail(CSM_ERR_INVALID_ARG, "empty vertex set");
    if (ne && (!src || !dst || !elabel)) return fail(CSM_ERR_INVALID_ARG, "null edge array");
    csm_status pst = prepare_tables(nv, vlabel, nullptr);
    const uint32_t nvl = (uint32_t)vlab_raw_.size(), nel = (uint32_t)elab_raw_.size();
    if (pst == CSM_OK) pst = build_lists(ne, src, dst, elabel, nvl, nel);
    // A load that fails part way leaves device tables half built: later calls are refused.
    if (pst != CSM_OK) poisoned_ = true;
    return pst;
}

// Label spaces, relations, candidate-rule specs, key layout and the device tables of a graph
// of nv vertices (raw vertex labels, or dense labels from a snapshot); allocates the list
// metadata.
csm_status Engine::prepare_tables(uint32_t nv, const uint32_t *vlabel, const uint8_t *vlab_dense) {
    CSM_CUDA(cudaSetDevice(device_));
    tables_ready_ = true;
    // Label spaces: the union of the labels of all queries (graph.cpp:389-433 keeps only
    // data labels that occur in the query).
    for (auto &q : queries_) {
        vlab_raw_.insert(vlab_raw_.end(), q.vlabel.begin(), q.vlabel.end());
        elab_raw_.insert(elab_raw_.end(), q.qe_elabel.begin(), q.qe_elabel.end());
    }
    std::sort(vlab_raw_.begin(), vlab_raw_.end());
    vlab_raw_.erase(std::unique(vlab_raw_.begin(), vlab_raw_.end()), vlab_raw_.end());
    std::sort(elab_raw_.begin(), elab_raw_.end());
    elab_raw_.erase(std::unique(elab_raw_.begin(), elab_raw_.end()), elab_raw_.end());
    if (vlab_raw_.size() >= CSM_NO_LABEL || elab_raw_.size() >= 255)
        return fail(CSM_ERR_LIMIT, "too many distinct labels across the registered queries");
    const uint32_t nvl = (uint32_t)vlab_raw_.size(), nel = (uint32_t)elab_raw_.size();
    auto vl = [&](uint32_t raw) {
        return (uint32_t)(std::lower_bound(vlab_raw_.begin(), vlab_raw_.end(), raw) - vlab_raw_.begin());
    };
    auto el = [&](uint32_t raw) {
        return (uint32_t)(std::lower_bound(elab_raw_.begin(), elab_raw_.end(), raw) - elab_raw_.begin());
    };
    // Relations: one per directed label triple of any query edge.
    rel_table_.assign((size_t)nvl * nel * nvl, CSM_NO_REL);
    auto rel_of_raw = [&](uint32_t a_raw, uint32_t l_raw, uint32_t b_raw) -> uint16_t {
        const size_t idx = ((size_t)vl(a_raw) * nel + el(l_raw)) * nvl + vl(b_raw);
        if (rel_table_[idx] == CSM_NO_REL) {
            rel_table_[idx] = (uint16_t)rel_triples_.size();
            rel_triples_.push_back((vl(a_raw) << 16) | (el(l_raw) << 8) | vl(b_raw));
        }
        return rel_table_[idx];
    };
    for (auto &q : queries_)
        for (uint32_t u = 0; u < q.nv; u++)
            for (auto &p : q.nbrs[u]) rel_of_raw(q.vlabel[u], p.second, q.vlabel[p.first]);
    if (rel_triples_.size() >= CSM_NO_REL) return fail(CSM_ERR_LIMIT, "too many relations");
    // NLF specs per dense label.
    std::vector<std::vector<NlfSpec>> by_label(nvl);
    nbitmaps_ = 0;
    for (auto &q : queries_) {
        nlf_base_.push_back(nbitmaps_);
        for (uint32_t u = 0; u < q.nv; u++) {
            NlfSpec sp{};
            sp.bitmap = nbitmaps_ + u;
            sp.ngroups = (uint32_t)q.nlf[u].size();
            for (uint32_t g = 0; g < sp.ngroups; g++) {
                sp.rel[g] = rel_of_raw(q.vlabel[u], q.nlf[u][g].elabel, q.nlf[u][g].vlabel);
                sp.cnt[g] = (uint16_t)q.nlf[u][g].count;
            }
            by_label[vl(q.vlabel[u])].push_back(sp);
        }
        nbitmaps_ += q.nv;
    }
    std::vector<uint32_t> spec_begin(nvl + 1, 0);
    std::vector<NlfSpec> specs;
    for (uint32_t a = 0; a < nvl; a++) {
        spec_begin[a] = (uint32_t)specs.size();
        specs.insert(specs.end(), by_label[a].begin(), by_label[a].end());
    }
    spec_begin[nvl] = (uint32_t)specs.size();

    g_.V = nv;
    g_.R = (uint32_t)rel_triples_.size();
    kl_.vbits = bits_for(nv ? nv - 1 : 0);
    kl_.rbits = bits_for(g_.R);
    if (kl_.end_bit() > 64) return fail(CSM_ERR_LIMIT, "vertex ids and relations do not fit a 64-bit batch key");
    words_ = (nv + 31) / 32;

    // Dense vertex labels.
    std::vector<uint8_t> vlab(nv, CSM_NO_LABEL);
    if (vlab_dense) {
        for (uint32_t v = 0; v < nv; v++)
            vlab[v] = vlab_dense[v] < nvl ? vlab_dense[v] : (uint8_t)CSM_NO_LABEL;
    } else {
        for (uint32_t v = 0; v < nv; v++) {
            auto it = std::lower_bound(vlab_raw_.begin(), vlab_raw_.end(), vlabel[v]);
            if (it != vlab_raw_.end() && *it == vlabel[v]) vlab[v] = (uint8_t)(it - vlab_raw_.begin());
        }
    }
    const size_t nmeta = (size_t)g_.R * nv;
    CSM_CUDA(dev_alloc(&g_.vlab, nv));
    CSM_CUDA(cudaMemcpy(g_.vlab, vlab.data(), nv, cudaMemcpyHostToDevice));
    CSM_CUDA(dev_alloc(&d_elab_raw_, nel));
    CSM_CUDA(cudaMemcpy(d_elab_raw_, elab_raw_.data(), sizeof(uint32_t) * nel, cudaMemcpyHostToDevice));
    CSM_CUDA(dev_alloc(&d_rel_table_, rel_table_.size()));
    CSM_CUDA(cudaMemcpy(d_rel_table_, rel_table_.data(), sizeof(uint16_t) * rel_table_.size(), cudaMemcpyHostToDevice));
    CSM_CUDA(dev_alloc(&d_spec_begin_, nvl + 1));
    CSM_CUDA(cudaMemcpy(d_spec_begin_, spec_begin.data(), sizeof(uint32_t) * (nvl + 1), cudaMemcpyHostToDevice));
    CSM_CUDA(dev_alloc(&d_specs_, specs.size()));
    if (!specs.empty())
        CSM_CUDA(cudaMemcpy(d_specs_, specs.data(), sizeof(NlfSpec) * specs.size(), cudaMemcpyHostToDevice));
    CSM_CUDA(dev_alloc(&d_bits_, (size_t)nbitmaps_ * words_));
    CSM_CUDA(cudaMemset(d_bits_, 0, sizeof(uint32_t) * (size_t)nbitmaps_ * words_));
    CSM_CUDA(dev_alloc(&g_.meta, nmeta));
    CSM_CUDA(dev_alloc(&g_.cap, nmeta));
    CSM_CUDA(dev_alloc(&g_.pool_top, 1));
    CSM_CUDA(dev_alloc(&d_touched_, words_));
    CSM_CUDA(cudaMemset(d_touched_, 0, sizeof(uint32_t) * words_));
    return CSM_OK;
}

// Initial lists from edge arrays, then the rest of the load.
csm_status Engine::build_lists(uint64_t ne, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                               uint32_t nvl, uint32_t nel) {
    // Edges -> keys -> sorted -> lists.
    const uint64_t m64 = 2 * ne;
    if (m64 >= 0x7FFFFFFFull) return fail(CSM_ERR_LIMIT, "too many initial edges for one load (limit 2^30)");
    const uint32_t m = (uint32_t)m64;
    uint32_t *d_src = nullptr, *d_dst = nullptr, *d_lab = nullptr;
    unsigned long long *k_raw = nullptr, *k_sorted = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
    LabelTables lt{d_elab_raw_, nel, d_rel_table_, nvl};
    csm_status st = CSM_OK;
    std::string berr;
    do {
        cudaError_t e;
        if ((e = dev_alloc(&d_src, ne)) || (e = dev_alloc(&d_dst, ne)) || (e = dev_alloc(&d_lab, ne)) ||
            (e = dev_alloc(&k_raw, m)) || (e = dev_alloc(&k_sorted, m))) {
            st = cuda_fail(e, "initial edge buffers");
            break;
        }
        if (ne) {
            cudaMemcpy(d_src, src, sizeof(uint32_t) * ne, cudaMemcpyHostToDevice);
            cudaMemcpy(d_dst, dst, sizeof(uint32_t) * ne, cudaMemcpyHostToDevice);
            cudaMemcpy(d_lab, elabel, sizeof(uint32_t) * ne, cudaMemcpyHostToDevice);
            store_build_keys(ne, d_src, d_dst, d_lab, nullptr, lt, g_, kl_, k_raw, stream_);
        }
        store_sort_keys(nullptr, temp_bytes, k_raw, k_sorted, m, kl_, stream_);
        if ((e = dev_alloc_bytes(&temp, temp_bytes + 16))) {
            st = cuda_fail(e, "sort scratch");
            break;
        }
        if (m) store_sort_keys(temp, temp_bytes, k_raw, k_sorted, m, kl_, stream_);
        cudaFree(d_src);
        cudaFree(d_dst);
        cudaFree(d_lab);
        d_src = d_dst = d_lab = nullptr;
        cudaFree(k_raw);
        k_raw = nullptr;
        // Pool: the laid-out lists plus room for batches; compaction regrows it later.
        const uint64_t max_batch = cfg_.max_batch ? cfg_.max_batch : (1ull << 20);
        unsigned long long want = cfg_.pool_entries ? cfg_.pool_entries
                                                    : (unsigned long long)(10 * m64 + 64 * max_batch + (1u << 20));
        if (want > 0xFFFFFFF0ull) want = 0xFFFFFFF0ull;
        g_.pool_cap = want;
        if ((e = dev_alloc(&g_.pool, g_.pool_cap))) {
            st = cuda_fail(e, "adjacency pool");
            break;
        }
        if ((e = store_build_from_keys(g_, k_sorted, m, kl_, stream_, berr))) {
            st = berr.empty() ? cuda_fail(e, "initial build") : fail(CSM_ERR_OOM, berr);
            break;
        }
    } while (false);
    cudaFree(d_src);
    cudaFree(d_dst);
    cudaFree(d_lab);
    cudaFree(k_raw);
    cudaFree(k_sorted);
    cudaFree(temp);
    if (st != CSM_OK) return st;
    return finish_load();
}

// Candidate bitmaps, planner statistics, plans and the per-batch buffers of a loaded graph.
csm_status Engine::finish_load() {
    // Candidate bitmaps, planner statistics, plans.
    NlfTables nt{d_spec_begin_, d_specs_, d_bits_, words_};
    store_nlf_all(g_, nt, stream_);
    std::vector<EdgeStats> stats;
    csm_status pst = compute_edge_stats(stats);
    if (pst != CSM_OK) return pst;
    pst = install_plans(stats);
    if (pst != CSM_OK) return pst;
    if (cfg_.replan_drift_pct > 0) {
        // Relation sizes at planning time, for the drift check after each batch.
        unsigned long long *d_sz = nullptr;
        CSM_CUDA(dev_alloc(&d_sz, g_.R));
        CSM_CUDA(cudaMemsetAsync(d_sz, 0, sizeof(unsigned long long) * g_.R, stream_));
        store_rel_sizes(g_, d_sz, stream_);
        std::vector<unsigned long long> h(g_.R);
        CSM_CUDA(cudaMemcpyAsync(h.data(), d_sz, sizeof(unsigned long long) * g_.R, cudaMemcpyDeviceToHost, stream_));
        CSM_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(d_sz);
        rel_size_.assign(h.begin(), h.end());
        rel_size_planned_ = rel_size_;
        CSM_CUDA(dev_alloc(&d_rel_delta_, g_.R));
        CSM_CUDA(cudaMallocHost(&h_rel_delta_, sizeof(long long) * g_.R));
    }
    const uint32_t np = (uint32_t)plans_.size();
    CSM_CUDA(dev_alloc(&d_seed_lo_, 3 * (size_t)np));
    CSM_CUDA(dev_alloc(&d_ticket_prefix_, np + 1));
    CSM_CUDA(dev_alloc(&d_counts_, 2 * (size_t)np));
    last_counts_.assign(2 * np, 0);
    cudaFreeHost(h_counts_);
    h_counts_ = nullptr;
    CSM_CUDA(cudaMallocHost(&h_counts_, sizeof(unsigned long long) * (2 * np + 32)));
    // Donation ring and the semi-BFS frontier.  The ring's slots are reused for the whole
    // launch, so it only needs room for the items in flight at once.
    CSM_CUDA(dev_alloc(&d_queue_, qcap_));
    CSM_CUDA(dev_alloc(&d_seq_, qcap_));
    CSM_CUDA(cudaMemset(d_seq_, 0, sizeof(unsigned long long) * qcap_));
    sc_.ctrl = d_ctrl_;
    sc_.queue = d_queue_;
    sc_.seq = d_seq_;
    sc_.qcap = qcap_;
    sc_.seed_lo = d_seed_lo_;
    sc_.ticket_prefix = d_ticket_prefix_;
    const unsigned long long fbytes = cfg_.frontier_bytes ? cfg_.frontier_bytes : (1ull << 30);
    frontier_cap_ = std::max<unsigned long long>(1024, fbytes / 2 / sizeof(WorkItem));
    if (opt_.search_strategy >= 2 || cfg_.autotune_batches > 0) {
        CSM_CUDA(dev_alloc(&d_frontier_[0], frontier_cap_));
        CSM_CUDA(dev_alloc(&d_frontier_[1], frontier_cap_));
    }
    if (cfg_.materialize_rows) {
        row_cap_ = cfg_.materialize_rows;
        CSM_CUDA(dev_alloc(&d_rows_, row_cap_ * CSM_ROW_WORDS));
    }
    csm_status bst = ensure_batch_capacity(cfg_.max_batch ? cfg_.max_batch : 65536);
    if (bst != CSM_OK) return bst;
    CSM_CUDA(cudaStreamSynchronize(stream_));
    CSM_CUDA(cudaGetLastError());
    unsigned long long top = 0;
    CSM_CUDA(cudaMemcpy(&top, g_.pool_top, sizeof(top), cudaMemcpyDeviceToHost));
    stats_.pool_used = top;
    stats_.pool_capacity = g_.pool_cap;
    graph_loaded_ = true;
    return CSM_OK;
}

// Planner statistics per directed query edge: candidate edges between the two endpoints'
// candidate sets and the average over sources (GetSummary, match_gpu.cu:589-609).
csm_status Engine::compute_edge_stats(std::vector<EdgeStats> &stats) {
    const uint32_t nvl = (uint32_t)vlab_raw_.size(), nel = (uint32_t)elab_raw_.size();
    auto vl = [&](uint32_t raw) {
        return (uint32_t)(std::lower_bound(vlab_raw_.begin(), vlab_raw_.end(), raw) - vlab_raw_.begin());
    };
    auto el = [&](uint32_t raw) {
        return (uint32_t)(std::lower_bound(elab_raw_.begin(), elab_raw_.end(), raw) - elab_raw_.begin());
    };
    unsigned long long *d_stat = nullptr;
    CSM_CUDA(dev_alloc(&d_stat, 2));
    stats.assign(queries_.size(), EdgeStats{});
    for (size_t qi = 0; qi < queries_.size(); qi++) {
        const Query &q = queries_[qi];
        stats[qi].card.assign(q.nv * q.nv, 0);
        stats[qi].avg.assign(q.nv * q.nv, 0.f);
        for (uint32_t u = 0; u < q.nv; u++)
            for (auto &p : q.nbrs[u]) {
                const uint32_t uu = p.first;
                const uint16_t rel = rel_table_[((size_t)vl(q.vlabel[u]) * nel + el(p.second)) * nvl + vl(q.vlabel[uu])];
                CSM_CUDA(cudaMemsetAsync(d_stat, 0, 16, stream_));
                store_edge_stats(g_, rel, d_bits_ + (size_t)(nlf_base_[qi] + u) * words_,
                                 d_bits_ + (size_t)(nlf_base_[qi] + uu) * words_, d_stat, stream_);
                unsigned long long h[2];
                CSM_CUDA(cudaMemcpyAsync(h, d_stat, 16, cudaMemcpyDeviceToHost, stream_));
                CSM_CUDA(cudaStreamSynchronize(stream_));
                stats[qi].card[u * q.nv + uu] = (uint32_t)std::min<unsigned long long>(h[0], 0xFFFFFFFFull);
                // GetSummary divides by the number of sources (match_gpu.cu:607), NaN when empty.
                stats[qi].avg[u * q.nv + uu] = (float)h[0] / (float)h[1];
            }
    }
    cudaFree(d_stat);
    return CSM_OK;
}

// Builds every query's plans from the statistics and uploads them (the plan count per query
// never changes; the tail-term array is regrown when a new plan set needs more terms).
csm_status Engine::install_plans(const std::vector<EdgeStats> &stats) {
    const uint32_t nvl = (uint32_t)vlab_raw_.size(), nel = (uint32_t)elab_raw_.size();
    auto vl = [&](uint32_t raw) {
        return (uint32_t)(std::lower_bound(vlab_raw_.begin(), vlab_raw_.end(), raw) - vlab_raw_.begin());
    };
    auto el = [&](uint32_t raw) {
        return (uint32_t)(std::lower_bound(elab_raw_.begin(), elab_raw_.end(), raw) - elab_raw_.begin());
    };
    std::vector<HostPlan> plans;
    std::vector<uint32_t> begin;
    for (size_t qi = 0; qi < queries_.size(); qi++) {
        const Query &q = queries_[qi];
        PlanOptions po;
        po.order = opt_.order;
        po.cartesian = opt_.cartesian;
        po.materialize = cfg_.materialize_rows > 0;
        auto rel_of = [&](uint32_t u, uint32_t uu) -> uint16_t {
            return rel_table_[((size_t)vl(q.vlabel[u]) * nel + el(q.edge_label(u, uu))) * nvl + vl(q.vlabel[uu])];
        };
        auto ps = build_plans(q, (uint16_t)qi, nlf_base_[qi], stats[qi], po, rel_of);
        begin.push_back((uint32_t)plans.size());
        plans.insert(plans.end(), ps.begin(), ps.end());
    }
    begin.push_back((uint32_t)plans.size());
    if (!plans_.empty() && plans.size() != plans_.size()) return fail(CSM_ERR_STATE, "re-planning changed the plan count");
    // Pendant plans with the same counting level and tail read one table: its entries do not
    // depend on the depths or on the query.  At most kMaxPendantTables tables (V entries each);
    // further pendant plans, or all of them when the tables do not fit, count normally.
    constexpr size_t kMaxPendantTables = 16;
    std::vector<std::vector<int64_t>> sigs;
    std::vector<uint32_t> memo_plan;
    for (uint32_t i = 0; i < plans.size(); i++) {
        DevPlan &dp = plans[i].dev;
        if (dp.memo_slot != CSM_MEMO_PENDING) continue;
        const DevLevel &lv = dp.lv[dp.tail_start - 1];
        const DevTail &t = dp.tail;
        std::vector<int64_t> sig{lv.bn_rel[0], lv.old_mask & 1, lv.nlf_bitmap, t.nkeys, t.nmasks, t.nclasses};
        for (int k = 0; k < t.nkeys; k++) sig.insert(sig.end(), {t.key_rel[k], t.key_old[k]});
        for (int k = 0; k < t.nmasks; k++) sig.push_back(t.mask[k]);
        for (int c = 0; c <= t.nclasses; c++) sig.push_back(t.class_term_begin[c]);
        for (const DevTailTerm &term : plans[i].terms) {
            sig.insert(sig.end(), {term.coef, term.nf});
            for (int j = 0; j < term.nf; j++) sig.push_back(term.f[j]);
        }
        size_t slot = std::find(sigs.begin(), sigs.end(), sig) - sigs.begin();
        if (slot == sigs.size()) {
            if (sigs.size() == kMaxPendantTables) continue;
            sigs.push_back(sig);
            memo_plan.push_back(i);
        }
        dp.memo_slot = (uint8_t)slot;
    }
    if (memo_plan.size() > memo_cap_) {
        if (d_memo_) cudaFree(d_memo_);
        d_memo_ = nullptr;
        memo_cap_ = 0;
        // The tables are an optimisation: they only take memory the adjacency pool is unlikely
        // to need (at most a quarter of what is free now).
        size_t free_b = 0, total_b = 0;
        const size_t want = memo_plan.size() * (size_t)g_.V * sizeof(unsigned long long);
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && want <= free_b / 4 &&
            dev_alloc(&d_memo_, memo_plan.size() * (size_t)g_.V) == cudaSuccess) {
            memo_cap_ = memo_plan.size();
        } else {
            (void)cudaGetLastError();
            d_memo_ = nullptr;
        }
    }
    if (memo_plan.size() > memo_cap_) {
        for (auto &hp : plans)
            if (hp.dev.memo_slot != CSM_NO_MEMO) hp.dev.memo_slot = CSM_MEMO_PENDING;
        memo_plan.clear();
    }
    memo_plan_ = std::move(memo_plan);
    std::vector<DevPlan> dplans;
    std::vector<DevTailTerm> terms;
    for (auto &hp : plans) {
        hp.dev.term_begin = (uint32_t)terms.size();
        terms.insert(terms.end(), hp.terms.begin(), hp.terms.end());
        dplans.push_back(hp.dev);
    }
    if (!d_plans_) CSM_CUDA(dev_alloc(&d_plans_, dplans.size()));
    CSM_CUDA(cudaMemcpyAsync(d_plans_, dplans.data(), sizeof(DevPlan) * dplans.size(), cudaMemcpyHostToDevice, stream_));
    if (terms.size() > terms_cap_ || !d_terms_) {
        if (d_terms_) cudaFree(d_terms_);
        d_terms_ = nullptr;
        terms_cap_ = std::max<size_t>(terms.size(), 1);
        CSM_CUDA(dev_alloc(&d_terms_, terms_cap_));
    }
    if (!terms.empty())
        CSM_CUDA(cudaMemcpyAsync(d_terms_, terms.data(), sizeof(DevTailTerm) * terms.size(), cudaMemcpyHostToDevice,
                                 stream_));
    CSM_CUDA(cudaStreamSynchronize(stream_));
    plans_ = std::move(plans);
    plan_begin_ = std::move(begin);
    // The kernel variant with the last-level intersection loop pays only where a plan ends
    // without a Cartesian tail (a last level the loop can count).
    last_loop_ = false;
    for (const auto &hp : plans_)
        if (hp.dev.tail_start == hp.dev.n && hp.dev.n >= 3) last_loop_ = true;
    return CSM_OK;
}

// Re-plans when a relation the plans read has grown or shrunk by more than the configured
// fraction since the plans were made (the reference plans once, technique_permutation.h:91-107).
csm_status Engine::maybe_replan() {
    bool drift = false;
    for (uint32_t r = 0; r < g_.R; r++) {
        rel_size_[r] += h_rel_delta_[r];
        const long long base = std::max<long long>(rel_size_planned_[r], 1024);
        const long long diff = rel_size_[r] - rel_size_planned_[r];
        if ((diff < 0 ? -diff : diff) * 100 > (long long)cfg_.replan_drift_pct * base) drift = true;
    }
    if (!drift) return CSM_OK;
    std::vector<EdgeStats> stats;
    csm_status st = compute_edge_stats(stats);
    if (st != CSM_OK) return st;
    st = install_plans(stats);
    if (st != CSM_OK) return st;
    rel_size_planned_ = rel_size_;
    clear_graphs();
    graph_gen_++;
    stats_.replans++;
    return CSM_OK;
}

// ---- Snapshots --------------------------------------------------------------------------
// File layout (little-endian): "CSMSNAP1", u32 version, u32 V, u32 R, u32 nqueries,
// u64 query fingerprint, u64 pool entries in use, u64 pool capacity, u8 dense vertex label[V],
// uint2 meta[R*V] (offset, size), u32 cap[R*V], u32 pool[in use].  Candidate bitmaps, plans and
// batch buffers are rebuilt on load; the lists keep their slack and layout.

namespace {
constexpr char kSnapMagic[8] = {'C', 'S', 'M', 'S', 'N', 'A', 'P', '1'};
constexpr uint32_t kSnapVersion = 1;

struct SnapHeader {
    char magic[8];
    uint32_t version, V, R, nqueries;
    uint64_t fingerprint, used, capacity;
};

struct FileCloser {
    FILE *f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};
}  // namespace

// FNV-1a over every query's vertex labels and labelled adjacency, in registration order: equal
// fingerprints mean equal relation numbering and list layout.
uint64_t Engine::query_fingerprint() const {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint32_t x) {
        for (int i = 0; i < 4; i++) {
            h ^= (x >> (8 * i)) & 0xFFu;
            h *= 1099511628211ull;
        }
    };
    mix((uint32_t)queries_.size());
    for (auto &q : queries_) {
        mix(q.nv);
        for (uint32_t u = 0; u < q.nv; u++) {
            mix(q.vlabel[u]);
            mix((uint32_t)q.nbrs[u].size());
            for (auto &p : q.nbrs[u]) {
                mix(p.first);
                mix(p.second);
            }
        }
    }
    return h;
}

csm_status Engine::save_snapshot(const char *path) {
    if (!path) return fail(CSM_ERR_INVALID_ARG, "null path");
    if (!graph_loaded_) return fail(CSM_ERR_STATE, "load the data graph first");
    if (poisoned_) return fail(CSM_ERR_STATE, "the engine failed an earlier call (see its error); recreate it");
    CSM_CUDA(cudaSetDevice(device_));
    CSM_CUDA(cudaStreamSynchronize(stream_));
    unsigned long long used = 0;
    CSM_CUDA(cudaMemcpy(&used, g_.pool_top, sizeof(used), cudaMemcpyDeviceToHost));
    const size_t nmeta = (size_t)g_.R * g_.V;
    std::vector<uint8_t> vlab(g_.V);
    std::vector<uint2> meta(nmeta);
    std::vector<uint32_t> cap(nmeta), pool(used);
    CSM_CUDA(cudaMemcpy(vlab.data(), g_.vlab, g_.V, cudaMemcpyDeviceToHost));
    CSM_CUDA(cudaMemcpy(meta.data(), g_.meta, sizeof(uint2) * nmeta, cudaMemcpyDeviceToHost));
    CSM_CUDA(cudaMemcpy(cap.data(), g_.cap, sizeof(uint32_t) * nmeta, cudaMemcpyDeviceToHost));
    if (used) CSM_CUDA(cudaMemcpy(pool.data(), g_.pool, sizeof(uint32_t) * used, cudaMemcpyDeviceToHost));
    SnapHeader h{};
    std::memcpy(h.magic, kSnapMagic, 8);
    h.version = kSnapVersion;
    h.V = g_.V;
    h.R = g_.R;
    h.nqueries = (uint32_t)queries_.size();
    h.fingerprint = query_fingerprint();
    h.used = used;
    h.capacity = g_.pool_cap;
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return fail(CSM_ERR_INVALID_ARG, std::string("cannot create ") + path);
    bool ok = std::fwrite(&h, sizeof(h), 1, fc.f) == 1 && std::fwrite(vlab.data(), 1, vlab.size(), fc.f) == vlab.size() &&
              std::fwrite(meta.data(), sizeof(uint2), nmeta, fc.f) == nmeta &&
              std::fwrite(cap.data(), sizeof(uint32_t), nmeta, fc.f) == nmeta &&
              std::fwrite(pool.data(), sizeof(uint32_t), used, fc.f) == used;
    ok = std::fflush(fc.f) == 0 && ok;
    if (!ok) return fail(CSM_ERR_INVALID_ARG, std::string("write failed: ") + path);
    return CSM_OK;
}

csm_status Engine::load_snapshot(const char *path) {
    if (!path) return fail(CSM_ERR_INVALID_ARG, "null path");
    if (graph_loaded_ || tables_ready_) return fail(CSM_ERR_STATE, "the data graph is already loaded");
    if (queries_.empty()) return fail(CSM_ERR_STATE, "register the snapshot's queries before loading it");
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return fail(CSM_ERR_INVALID_ARG, std::string("cannot open ") + path);
    SnapHeader h{};
    if (std::fread(&h, sizeof(h), 1, fc.f) != 1 || std::memcmp(h.magic, kSnapMagic, 8) != 0 || h.version != kSnapVersion)
        return fail(CSM_ERR_INVALID_ARG, "not a snapshot of this format");
    if (h.nqueries != queries_.size() || h.fingerprint != query_fingerprint())
        return fail(CSM_ERR_INVALID_ARG, "the snapshot was taken with other queries");
    if (h.V == 0 || h.used > h.capacity || h.capacity > 0xFFFFFFF0ull)
        return fail(CSM_ERR_INVALID_ARG, "corrupt snapshot header");
    // Everything is read and validated before any device table is built, so a rejected file
    // leaves the engine as it was (a good snapshot or load_graph may follow).
    std::vector<uint8_t> vlab(h.V);
    if (std::fread(vlab.data(), 1, h.V, fc.f) != h.V) return fail(CSM_ERR_INVALID_ARG, "truncated snapshot");
    if (h.R == 0 || (uint64_t)h.R * h.V > (1ull << 36)) return fail(CSM_ERR_INVALID_ARG, "corrupt snapshot header");
    const size_t nmeta = (size_t)h.R * h.V;
    std::vector<uint2> meta(nmeta);
    std::vector<uint32_t> cap(nmeta), pool(h.used);
    if (std::fread(meta.data(), sizeof(uint2), nmeta, fc.f) != nmeta ||
        std::fread(cap.data(), sizeof(uint32_t), nmeta, fc.f) != nmeta ||
        std::fread(pool.data(), sizeof(uint32_t), h.used, fc.f) != h.used)
        return fail(CSM_ERR_INVALID_ARG, "truncated snapshot");
    for (size_t i = 0; i < nmeta; i++)
        if ((uint64_t)meta[i].x + cap[i] > h.used || meta[i].y > cap[i])
            return fail(CSM_ERR_INVALID_ARG, "corrupt snapshot list table");
    // Every live entry must name a vertex of the graph, carry no batch flag, and the lists must
    // be strictly ascending: the kernels index by these ids and search these lists.
    for (size_t i = 0; i < nmeta; i++) {
        const uint32_t *l = pool.data() + meta[i].x;
        for (uint32_t j = 0; j < meta[i].y; j++)
            if ((l[j] >> 1) >= h.V || (l[j] & 1u) || (j && l[j] <= l[j - 1]))
                return fail(CSM_ERR_INVALID_ARG, "corrupt snapshot adjacency list");
    }
    csm_status st = prepare_tables(h.V, nullptr, vlab.data());
    if (st == CSM_OK && g_.R != h.R)  // equal fingerprints give equal relations
        st = fail(CSM_ERR_INVALID_ARG, "the snapshot's relations differ from the queries'");
    if (st == CSM_OK) st = upload_snapshot(h.used, h.capacity, meta, cap, pool);
    if (st != CSM_OK) poisoned_ = true;
    return st;
}

// Device side of load_snapshot: the pool, the list table and the entries in use.
csm_status Engine::upload_snapshot(uint64_t used, uint64_t capacity, const std::vector<uint2> &meta,
                                   const std::vector<uint32_t> &cap, const std::vector<uint32_t> &pool) {
    const size_t nmeta = meta.size();
    const uint64_t max_batch = cfg_.max_batch ? cfg_.max_batch : (1ull << 20);
    unsigned long long want = cfg_.pool_entries ? cfg_.pool_entries : capacity;
    want = std::max<unsigned long long>(want, used + 64 * max_batch + (1u << 20));
    if (want > 0xFFFFFFF0ull) want = 0xFFFFFFF0ull;
    g_.pool_cap = want;
    CSM_CUDA(dev_alloc(&g_.pool, g_.pool_cap));
    CSM_CUDA(cudaMemcpy(g_.meta, meta.data(), sizeof(uint2) * nmeta, cudaMemcpyHostToDevice));
    CSM_CUDA(cudaMemcpy(g_.cap, cap.data(), sizeof(uint32_t) * nmeta, cudaMemcpyHostToDevice));
    if (used) CSM_CUDA(cudaMemcpy(g_.pool, pool.data(), sizeof(uint32_t) * used, cudaMemcpyHostToDevice));
    const unsigned long long top = used;
    CSM_CUDA(cudaMemcpy(g_.pool_top, &top, sizeof(top), cudaMemcpyHostToDevice));
    return finish_load();
}

csm_status Engine::ensure_batch_capacity(uint64_t n) {
    if (n <= batch_cap_) return CSM_OK;
    uint64_t cap = std::max<uint64_t>(n, batch_cap_ * 2);
    if (2 * cap >= 0x7FFFFFFFull) return fail(CSM_ERR_LIMIT, "batch too large (limit 2^30 updates)");
    const size_t m = 2 * cap;
    // The new buffers are allocated first and replace the old ones only when all exist: a
    // failed growth leaves the engine working at its previous capacity.
    uint32_t *upd_src = nullptr, *upd_dst = nullptr, *upd_lab = nullptr, *pin = nullptr;
    uint8_t *upd_del = nullptr;
    unsigned long long *keys_raw = nullptr, *keys = nullptr;
    void *sort_temp = nullptr;
    BatchScratch b;
    size_t tb = 0;
    store_sort_keys(nullptr, tb, nullptr, nullptr, (uint32_t)m, kl_, stream_);
    cudaError_t e;
    if ((e = dev_alloc(&upd_src, cap)) || (e = dev_alloc(&upd_dst, cap)) || (e = dev_alloc(&upd_lab, cap)) ||
        (e = dev_alloc(&upd_del, cap)) || (e = cudaMallocHost(&pin, sizeof(uint32_t) * 3 * cap + cap + 64)) ||
        (e = dev_alloc(&keys_raw, m)) || (e = dev_alloc(&keys, m)) || (e = dev_alloc_bytes(&sort_temp, tb + 16)) ||
        (e = dev_alloc(&b.eff, m)) || (e = dev_alloc(&b.heads, m)) || (e = dev_alloc(&b.nheads, 1)) ||
        (e = dev_alloc(&b.seg_nins, m)) || (e = dev_alloc(&b.seg_ndel, m)) || (e = dev_alloc(&b.seg_end, m)) ||
        (e = dev_alloc(&b.scr_y, m)) || (e = dev_alloc(&b.scr_lb, m)) || (e = dev_alloc(&b.counters, 2)) ||
        (e = dev_alloc(&b.error, 1))) {
        void *got[] = {upd_src, upd_dst, upd_lab, upd_del, keys_raw, keys, sort_temp, b.eff, b.heads, b.nheads,
                       b.seg_nins, b.seg_ndel, b.seg_end, b.scr_y, b.scr_lb, b.counters, b.error};
        for (void *p : got)
            if (p) cudaFree(p);
        if (pin) cudaFreeHost(pin);
        cudaGetLastError();
        return cuda_fail(e, "batch buffers");
    }
    CSM_CUDA(cudaStreamSynchronize(stream_));
    clear_graphs();
    graph_gen_++;
    void *old[] = {d_upd_src_, d_upd_dst_, d_upd_lab_, d_upd_del_, d_keys_raw_, d_keys_, d_sort_temp_, bs_.eff,
                   bs_.heads, bs_.nheads, bs_.seg_nins, bs_.seg_ndel, bs_.seg_end, bs_.scr_y, bs_.scr_lb, bs_.counters,
                   bs_.error};
    for (void *p : old)
        if (p) cudaFree(p);
    if (h_pin_) cudaFreeHost(h_pin_);
    d_upd_src_ = upd_src;
    d_upd_dst_ = upd_dst;
    d_upd_lab_ = upd_lab;
    d_upd_del_ = upd_del;
    h_pin_ = pin;
    d_keys_raw_ = keys_raw;
    d_keys_ = keys;
    d_sort_temp_ = sort_temp;
    sort_temp_bytes_ = tb;
    bs_ = b;
    batch_cap_ = cap;
    return CSM_OK;
}

csm_status Engine::apply_host(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                              const uint8_t *is_delete, csm_batch_result *out) {
    return apply_host_on(stream_, n, src, dst, elabel, is_delete, out);
}

csm_status Engine::apply_host_ctx(const ExecContext &ctx, uint64_t n, const uint32_t *src, const uint32_t *dst,
                                  const uint32_t *elabel, const uint8_t *is_delete, csm_batch_result *out) {
    if (ctx.frontier_cap && (!ctx.frontier[0] || !ctx.frontier[1]))
        return fail(CSM_ERR_INVALID_ARG, "frontier buffers missing");
    const EnumScratch saved = sc_;
    WorkItem *f0 = d_frontier_[0], *f1 = d_frontier_[1];
    const unsigned long long fcap = frontier_cap_;
    sc_ = ctx.scratch;
    d_frontier_[0] = ctx.frontier[0];
    d_frontier_[1] = ctx.frontier[1];
    frontier_cap_ = ctx.frontier_cap;
    const csm_status st = apply_host_on(ctx.stream ? ctx.stream : stream_, n, src, dst, elabel, is_delete, out);
    sc_ = saved;
    d_frontier_[0] = f0;
    d_frontier_[1] = f1;
    frontier_cap_ = fcap;
    return st;
}

csm_status Engine::apply_host_on(cudaStream_t s, uint64_t n, const uint32_t *src, const uint32_t *dst,
                                 const uint32_t *elabel, const uint8_t *is_delete, csm_batch_result *out) {
    if (!graph_loaded_) return fail(CSM_ERR_STATE, "load the data graph first");
    if (poisoned_) return fail(CSM_ERR_STATE, "the engine failed an earlier call (see its error); recreate it");
    if (n && (!src || !dst || !elabel)) return fail(CSM_ERR_INVALID_ARG, "null update array");
    csm_status st = ensure_batch_capacity(n);
    if (st != CSM_OK) return st;
    bool has_delete = false;
    if (is_delete)
        for (uint64_t i = 0; i < n && !has_delete; i++) has_delete = is_delete[i] != 0;
    // Timed from the first host->device copy (technique_permutation.h:123 includes the H2D).
    CSM_CUDA(cudaEventRecord(ev_[0], s));
    if (n) {
        CSM_CUDA(cudaMemcpyAsync(d_upd_src_, src, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
        CSM_CUDA(cudaMemcpyAsync(d_upd_dst_, dst, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
        CSM_CUDA(cudaMemcpyAsync(d_upd_lab_, elabel, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
        if (has_delete)
            CSM_CUDA(cudaMemcpyAsync(d_upd_del_, is_delete, n, cudaMemcpyHostToDevice, s));
    }
    return run_batch(n, d_upd_src_, d_upd_dst_, d_upd_lab_, has_delete ? d_upd_del_ : nullptr, has_delete, s, out);
}

csm_status Engine::apply_device(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                                const uint8_t *is_delete, cudaStream_t stream, csm_batch_result *out) {
    if (!graph_loaded_) return fail(CSM_ERR_STATE, "load the data graph first");
    if (poisoned_) return fail(CSM_ERR_STATE, "the engine failed an earlier call (see its error); recreate it");
    if (n && (!src || !dst || !elabel)) return fail(CSM_ERR_INVALID_ARG, "null update array");
    csm_status st = ensure_batch_capacity(n);
    if (st != CSM_OK) return st;
    cudaStream_t s = stream ? stream : stream_;
    CSM_CUDA(cudaEventRecord(ev_[0], s));
    if (graphs_on() && n) {
        // The replayed graph reads the engine's own update buffers.
        CSM_CUDA(cudaMemcpyAsync(d_upd_src_, src, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        CSM_CUDA(cudaMemcpyAsync(d_upd_dst_, dst, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        CSM_CUDA(cudaMemcpyAsync(d_upd_lab_, elabel, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
        if (is_delete) CSM_CUDA(cudaMemcpyAsync(d_upd_del_, is_delete, n, cudaMemcpyDeviceToDevice, s));
        return run_batch(n, d_upd_src_, d_upd_dst_, d_upd_lab_, is_delete ? d_upd_del_ : nullptr, is_delete != nullptr,
                         s, out);
    }
    return run_batch(n, src, dst, elabel, is_delete, is_delete != nullptr, s, out);
}

csm_status Engine::apply_device_noalloc(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                                        const uint8_t *is_delete, cudaStream_t stream, const EnumScratch &scratch,
                                        csm_batch_result *out) {
    if (!graph_loaded_) return fail(CSM_ERR_STATE, "load the data graph first");
    if (poisoned_) return fail(CSM_ERR_STATE, "the engine failed an earlier call (see its error); recreate it");
    if (n && (!src || !dst || !elabel)) return fail(CSM_ERR_INVALID_ARG, "null update array");
    if (n > batch_cap_)
        return fail(CSM_ERR_LIMIT, "batch of " + std::to_string(n) + " updates exceeds the " +
                                       std::to_string(batch_cap_) +
                                       " preallocated at load time (csm_config.max_batch); this call does not grow it");
    // This call never compacts or grows the adjacency pool: refuse, before anything changes, a
    // batch that could need more room than is free (the headroom compaction keeps elsewhere).
    const unsigned long long headroom = 64ull * n + (1u << 20);
    if (stats_.pool_used + headroom > g_.pool_cap)
        return fail(CSM_ERR_LIMIT, "the adjacency pool has " + std::to_string(g_.pool_cap - std::min<unsigned long long>(
                                                                                      stats_.pool_used, g_.pool_cap)) +
                                       " free entries, fewer than the " + std::to_string(headroom) +
                                       " this batch may need; this call never compacts the pool: apply a batch "
                                       "through csm_apply_batch_device, or size pool_entries for the stream");
    cudaStream_t s = stream ? stream : stream_;
    CSM_CUDA(cudaEventRecord(ev_[0], s));
    const EnumScratch saved = sc_;
    sc_ = scratch;
    no_alloc_ = true;
    const csm_status st = run_batch(n, src, dst, elabel, is_delete, is_delete != nullptr, s, out);
    no_alloc_ = false;
    sc_ = saved;
    return st;
}

csm_status Engine::enqueue_batch(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                                 const uint8_t *is_delete, bool has_delete, bool tuning, cudaStream_t s) {
    const uint32_t m = (uint32_t)(2 * n);
    const uint32_t np = (uint32_t)plans_.size();
    CSM_CUDA(cudaMemsetAsync(bs_.nheads, 0, sizeof(unsigned int), s));
    CSM_CUDA(cudaMemsetAsync(bs_.counters, 0, 2 * sizeof(unsigned long long), s));
    CSM_CUDA(cudaMemsetAsync(bs_.error, 0, sizeof(unsigned int), s));
    CSM_CUDA(cudaMemsetAsync(d_counts_, 0, 2 * sizeof(unsigned long long) * np, s));
    NlfTables nt{d_spec_begin_, d_specs_, d_bits_, words_};
    if (m) {
        LabelTables lt{d_elab_raw_, (uint32_t)elab_raw_.size(), d_rel_table_, (uint32_t)vlab_raw_.size()};
        store_build_keys(n, src, dst, elabel, is_delete, lt, g_, kl_, d_keys_raw_, s);
        size_t tb = sort_temp_bytes_;
        CSM_CUDA(store_sort_keys(d_sort_temp_, tb, d_keys_raw_, d_keys_, m, kl_, s));
        store_classify(m, d_keys_, kl_, g_, bs_, s);
        store_touched(m, d_keys_, kl_, d_touched_, words_, s);
        stats_.kernel_launches += 4;
        if (d_rel_delta_) {
            CSM_CUDA(cudaMemsetAsync(d_rel_delta_, 0, sizeof(long long) * g_.R, s));
            store_rel_delta(m, d_keys_, kl_, bs_, d_rel_delta_, s);
            stats_.kernel_launches++;
        }
        if (has_delete) {
            // Destroyed embeddings are counted on the graph before the deletions, with the
            // deleted edges flagged; then the flagged entries are compacted away.
            csm_status st = enumerate_phase(CSM_PHASE_DEL, m, s);
            if (st != CSM_OK) return st;
            store_delete(m, d_keys_, kl_, g_, bs_, s);
            stats_.kernel_launches++;
        }
        store_insert(m, d_keys_, kl_, g_, bs_, s);
        store_nlf_update(m, d_keys_, kl_, g_, bs_, nt, s);
        stats_.kernel_launches += 2;
        csm_status st = CSM_OK;
        if (tuning) {
            // Autotuning: the insertion phase runs once per candidate configuration (it does
            // not change the graph, so every run counts the same matches); each run is timed.
            const LaunchConfig keep = lc_;
            for (size_t c = 0; c < tune_cands_.size(); c++) {
                set_launch_config(tune_cands_[c]);
                CSM_CUDA(cudaMemsetAsync(d_counts_ + np, 0, sizeof(unsigned long long) * np, s));
                CSM_CUDA(cudaEventRecord(tune_ev_[2 * c], s));
                st = enumerate_phase(CSM_PHASE_INS, m, s);
                if (st != CSM_OK) return st;
                CSM_CUDA(cudaEventRecord(tune_ev_[2 * c + 1], s));
            }
            set_launch_config(keep);
            tuned_this_batch_ = true;
        } else {
            st = enumerate_phase(CSM_PHASE_INS, m, s);
            if (st != CSM_OK) return st;
        }
        store_clear_ins(m, d_keys_, kl_, g_, bs_, s);
        stats_.kernel_launches++;
    }
    return enqueue_readback(s);
}

// The end of a batch's device work: the timing event and the copies the host reads after the
// batch's single synchronisation (counts, edge counters, pool top, error bits).
csm_status Engine::enqueue_readback(cudaStream_t s) {
    const uint32_t np = (uint32_t)plans_.size();
    unsigned int *h_err = reinterpret_cast<unsigned int *>(h_counts_ + 2 * np + 3);
    CSM_CUDA(record_event(ev_[1], s));
    CSM_CUDA(cudaMemcpyAsync(h_counts_, d_counts_, 2 * sizeof(unsigned long long) * np, cudaMemcpyDeviceToHost, s));
    CSM_CUDA(cudaMemcpyAsync(h_counts_ + 2 * np, bs_.counters, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s));
    CSM_CUDA(cudaMemcpyAsync(h_counts_ + 2 * np + 2, g_.pool_top, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             s));
    CSM_CUDA(cudaMemcpyAsync(h_err, bs_.error, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    if (d_rel_delta_)
        CSM_CUDA(cudaMemcpyAsync(h_rel_delta_, d_rel_delta_, sizeof(long long) * g_.R, cudaMemcpyDeviceToHost, s));
    return CSM_OK;
}

// Replays the batch's device work from a CUDA graph captured for this batch size and launch
// configuration (captured on first use; any reallocation of engine buffers starts a new one).
csm_status Engine::launch_graph(uint64_t n, bool has_delete, cudaStream_t s) {
    GraphKey key{n, has_delete, graph_gen_, lc_.strategy, lc_.steal_chunk, lc_.warps_per_block, lc_.occupancy, blocks_};
    GraphEntry *hit = nullptr;
    for (auto &g : graphs_)
        if (g.key == key) hit = &g;
    if (!hit) {
        if (graphs_.size() >= 8) clear_graphs();
        const Stats0 before{stats_.kernel_launches, stats_.enum_launches};
        CSM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        capturing_ = true;
        const csm_status st = enqueue_batch(n, d_upd_src_, d_upd_dst_, d_upd_lab_, has_delete ? d_upd_del_ : nullptr,
                                            has_delete, false, s);
        capturing_ = false;
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s, &g);
        if (st != CSM_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        GraphEntry e;
        e.key = key;
        const cudaError_t ie = cudaGraphInstantiate(&e.exec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
        e.kernels = stats_.kernel_launches - before.kernels;
        e.enum_launches = stats_.enum_launches - before.enum_launches;
        stats_.kernel_launches = before.kernels;
        stats_.enum_launches = before.enum_launches;
        graphs_.push_back(e);
        hit = &graphs_.back();
    }
    CSM_CUDA(cudaGraphLaunch(hit->exec, s));
    stats_.kernel_launches += hit->kernels;
    stats_.enum_launches += hit->enum_launches;
    stats_.graph_launches++;
    if (n) phase_ran_[1] = true;
    if (n && has_delete) phase_ran_[0] = true;
    return CSM_OK;
}

void Engine::clear_graphs() {
    for (auto &g : graphs_)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
}

csm_status Engine::run_batch(uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                             const uint8_t *is_delete, bool has_delete, cudaStream_t s, csm_batch_result *out) {
    const uint32_t m = (uint32_t)(2 * n);
    const uint32_t np = (uint32_t)plans_.size();
    rows_valid_ = false;
    phase_ran_[0] = phase_ran_[1] = false;
    last_frontier_rows_ = 0;
    deferred_ = CSM_OK;
    NlfTables nt{d_spec_begin_, d_specs_, d_bits_, words_};
    const bool tuning = tune_left_ > 0 && !no_alloc_ && cfg_.materialize_rows == 0;
    csm_status est;
    if (graphs_on() && !tuning && src == d_upd_src_)
        est = launch_graph(n, has_delete, s);
    else
        est = enqueue_batch(n, src, dst, elabel, is_delete, has_delete, tuning, s);
    if (est != CSM_OK) {
        // The batch's device work stopped part way (a CUDA failure): the graph may hold part
        // of it, so the engine refuses later batches.
        poisoned_ = true;
        return est;
    }
    unsigned int *h_err = reinterpret_cast<unsigned int *>(h_counts_ + 2 * np + 3);
    for (int attempt = 0;; attempt++) {
        if (attempt > 0) {
            const csm_status rb = enqueue_readback(s);
            if (rb != CSM_OK) return rb;
        }
        CSM_CUDA(cudaStreamSynchronize(s));
        CSM_CUDA(cudaGetLastError());
        stats_.pool_used = h_counts_[2 * np + 2];
        if (!(*h_err & CSM_ERRBIT_POOL)) break;
        if (attempt > 0) {
            poisoned_ = true;
            return fail(CSM_ERR_OOM, "adjacency pool exhausted while applying a batch");
        }
        // The pool ran out during the merge, and the insertion phase skipped its work: lay the
        // lists out again in a larger pool, redo the merge (lists already merged are skipped),
        // the candidate refresh and the insertion phase.
        if (no_alloc_) {
            poisoned_ = true;
            return fail(CSM_ERR_OOM, "adjacency pool exhausted in a call that may not allocate; size pool_entries "
                                     "for the stream or apply batches through csm_apply_batch");
        }
        stats_.pool_used = g_.pool_cap;
        csm_status cst = maybe_compact(s);
        if (cst != CSM_OK) {
            poisoned_ = true;  // this batch's lists are only partly merged
            return cst;
        }
        CSM_CUDA(cudaMemsetAsync(bs_.error, 0, sizeof(unsigned int), s));
        CSM_CUDA(cudaMemsetAsync(d_counts_ + np, 0, sizeof(unsigned long long) * np, s));
        store_insert(m, d_keys_, kl_, g_, bs_, s);
        store_nlf_update(m, d_keys_, kl_, g_, bs_, nt, s);
        csm_status st = enumerate_phase(CSM_PHASE_INS, m, s);
        if (st != CSM_OK) return st;
        store_clear_ins(m, d_keys_, kl_, g_, bs_, s);
    }
    float total_ms = 0.f, enum_ms = 0.f;
    CSM_CUDA(cudaEventElapsedTime(&total_ms, ev_[0], ev_[1]));
    if (tuned_this_batch_) {
        tuned_this_batch_ = false;
        for (size_t c = 0; c < tune_cands_.size(); c++) {
            float t = 0.f;
            CSM_CUDA(cudaEventElapsedTime(&t, tune_ev_[2 * c], tune_ev_[2 * c + 1]));
            tune_ms_[c] += t;
        }
        if (--tune_left_ == 0) {
            size_t best = 0;
            for (size_t c = 1; c < tune_cands_.size(); c++)
                if (tune_ms_[c] < tune_ms_[best]) best = c;
            set_launch_config(tune_cands_[best]);
        }
    }
    for (int ph = 0; ph < 2; ph++) {
        if (!phase_ran_[ph]) continue;
        float t = 0.f;
        CSM_CUDA(cudaEventElapsedTime(&t, ev_[2 + 2 * ph], ev_[3 + 2 * ph]));
        enum_ms += t;
        const EnumControl &c = h_ctrl_[ph];
        stats_.enum_scan_entries += c.scan_entries;
        stats_.enum_probes += c.probes;
        stats_.enum_tail_lists += c.tail_lists;
        stats_.donations += c.donations;
        stats_.donations_refused += c.queue_full;
        stats_.enum_shared_last += c.shared_last;
        if (c.error & CSM_ERRBIT_CORRUPT) {
            poisoned_ = true;
            return fail(CSM_ERR_STATE, describe_bad(c));
        }
        // A launch that ran past its time limit stopped early; the graph still holds the whole
        // batch (the update kernels do not depend on the counts), so only the counts are short.
        if ((c.error & CSM_ERRBIT_TIMEOUT) && deferred_ == CSM_OK)
            deferred_ = fail(CSM_ERR_TIMEOUT, "the enumeration ran past its time limit (time_limit_us): this batch's "
                                              "counts are incomplete; the graph holds the whole batch");
        if ((c.error & CSM_ERRBIT_OUTPUT) && deferred_ == CSM_OK)
            deferred_ = fail(CSM_ERR_OVERFLOW, "embedding row buffer too small");
    }
    for (uint32_t i = 0; i < 2 * np; i++) last_counts_[i] = h_counts_[i];
    const uint64_t ins = h_counts_[2 * np], del = h_counts_[2 * np + 1];
    stats_.batches++;
    stats_.enum_ns += (uint64_t)(enum_ms * 1e6);
    stats_.apply_ns += (uint64_t)((total_ms - enum_ms) * 1e6);
    if (out) {
        for (uint32_t qi = 0; qi < queries_.size(); qi++) {
            csm_batch_result &r = out[qi];
            std::memset(&r, 0, sizeof(r));
            for (uint32_t p = plan_begin_[qi]; p < plan_begin_[qi + 1]; p++) {
                r.positive += last_counts_[p + np];
                r.negative += last_counts_[p];
            }
            r.inserted = ins;
            r.deleted = del;
            r.latency_ns = (uint64_t)(total_ms * 1e6);
            r.enum_ns = (uint64_t)(enum_ms * 1e6);
            r.apply_ns = r.latency_ns > r.enum_ns ? r.latency_ns - r.enum_ns : 0;
        }
    }
    if (cfg_.materialize_rows) rows_valid_ = deferred_ == CSM_OK;
    if (no_alloc_) return deferred_;
    if (d_rel_delta_ && m) {
        const csm_status rst = maybe_replan();
        if (rst != CSM_OK) return rst;
    }
    // The batch is applied: a compaction that cannot run now (no memory for the new layout) is
    // retried after the next batch, and a pool that then overflows takes the rerun path.
    if (maybe_compact(s) != CSM_OK && poisoned_) return CSM_ERR_CUDA;
    return deferred_;
}

csm_status Engine::enumerate_phase(uint32_t phase, uint32_t m, cudaStream_t s) {
    const uint32_t np = (uint32_t)plans_.size();
    const uint32_t total_warps = (uint32_t)(blocks_ * warps_per_block_);
    EnumParams P{};
    P.plans = d_plans_;
    P.nplans = np;
    P.terms = d_terms_;
    P.g = g_.view();
    P.bits = d_bits_;
    P.words = words_;
    P.keys = d_keys_;
    P.m = m;
    P.kl = kl_;
    P.eff = bs_.eff;
    P.seg_flagged = phase == CSM_PHASE_INS ? bs_.seg_nins : bs_.seg_ndel;
    P.phase = phase;
    P.seed_lo = sc_.seed_lo;
    P.ticket_prefix = sc_.ticket_prefix;
    P.queue = sc_.queue;
    P.seq = sc_.seq;
    P.qmask = sc_.qcap - 1;
    P.ctrl = sc_.ctrl;
    P.counts = d_counts_ + (phase == CSM_PHASE_INS ? np : 0);
    P.steal_min = lc_.steal_chunk;
    // An idle warp leaves as soon as no warp holds work; the bound (seconds of polling) only
    // ends the wait if that never happens.
    P.idle_limit = 1u << 24;
    P.time_limit_ns = time_limit_us_ * 1000ull;
    P.abort_flag = phase == CSM_PHASE_INS ? bs_.error : nullptr;
    P.touched = d_touched_;
    P.last_loop = last_loop_ ? 1u : 0u;
    P.rows = d_rows_;
    P.row_cap = row_cap_;
    const bool rows = cfg_.materialize_rows > 0;
    const int strategy = lc_.strategy;
    const int ph = phase == CSM_PHASE_INS ? 1 : 0;
    phase_ran_[ph] = true;
    CSM_CUDA(record_event(ev_[2 + 2 * ph], s));

    launch_ctrl_reset(sc_.ctrl, 0, 0, s);
    launch_seed_tickets(d_plans_, np, d_keys_, m, kl_, sc_.seed_lo, sc_.ticket_prefix, sc_.ctrl, s);
    stats_.kernel_launches += 3;
    const WorkItem *frontier = nullptr;
    unsigned long long nfront = 0;
    if (strategy >= 2 && !rows) {
        // Semi-BFS (Matching / BfsMatching, match_gpu.cu:1916-2294): expand levels while the
        // frontier is small (strategy 2) or while it fits the budget (strategy 3); the size of
        // the next level is bounded from list sizes before it is written, so a level that would
        // not fit is never started and the search continues depth first from the current one.
        CSM_CUDA(cudaMemcpyAsync(h_counts_ + 2 * np + 4, &sc_.ctrl->nticket, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
        CSM_CUDA(cudaStreamSynchronize(s));
        unsigned long long cur = h_counts_[2 * np + 4] * 32;  // seed candidates (upper bound)
        const unsigned long long target = (unsigned long long)lc_.frontier_mult * total_warps;
        int buf = 0;
        for (int level = 0; level < CSM_MAXQV; level++) {
            if (strategy == 2 && cur >= target) break;
            if (cur == 0) break;
            unsigned long long bound = cur;
            if (frontier) {
                h_counts_[2 * np + 4] = nfront;
                CSM_CUDA(cudaMemcpyAsync(d_misc_, h_counts_ + 2 * np + 4, 8, cudaMemcpyHostToDevice, s));
                CSM_CUDA(cudaMemsetAsync(&sc_.ctrl->expand_bound, 0, 8, s));
                launch_expand_bound(P, frontier, d_misc_, s);
                CSM_CUDA(cudaMemcpyAsync(h_counts_ + 2 * np + 5, &sc_.ctrl->expand_bound, 8, cudaMemcpyDeviceToHost, s));
                CSM_CUDA(cudaStreamSynchronize(s));
                bound = h_counts_[2 * np + 5];
            }
            if (bound > frontier_cap_) break;
            EnumParams X = P;
            X.mode = CSM_ENUM_MODE_EXPAND;
            X.donate = 0;
            X.frontier = frontier;
            X.expand_out = d_frontier_[buf];
            X.expand_cap = frontier_cap_;
            if (frontier) launch_ctrl_reset(sc_.ctrl, 0, nfront, s);
            launch_enumerate(X, blocks_, warps_per_block_, occupancy_, s);
            stats_.enum_launches++;
            stats_.kernel_launches++;
            CSM_CUDA(cudaMemcpyAsync(&h_ctrl_[ph], sc_.ctrl, sizeof(EnumControl), cudaMemcpyDeviceToHost, s));
            CSM_CUDA(cudaStreamSynchronize(s));
            const unsigned long long rows_out = h_ctrl_[ph].out_rows;
            const unsigned int errb = h_ctrl_[ph].error;
            if (errb & (CSM_ERRBIT_OUTPUT | CSM_ERRBIT_TIMEOUT | CSM_ERRBIT_CORRUPT)) {
                // Out of time (or, never expected, of frontier room): the phase stops here and
                // the batch reports it; the update kernels after it still run.
                if ((errb & CSM_ERRBIT_OUTPUT) && deferred_ == CSM_OK)
                    deferred_ = fail(CSM_ERR_OVERFLOW, "semi-BFS frontier overflow");
                CSM_CUDA(record_event(ev_[3 + 2 * ph], s));
                return CSM_OK;
            }
            // This expansion launch's work counters, before the next launch's control block
            // replaces them (the batch's final launch is added when the batch completes).
            stats_.enum_scan_entries += h_ctrl_[ph].scan_entries;
            stats_.enum_probes += h_ctrl_[ph].probes;
            stats_.enum_tail_lists += h_ctrl_[ph].tail_lists;
            stats_.donations += h_ctrl_[ph].donations;
            stats_.donations_refused += h_ctrl_[ph].queue_full;
            stats_.enum_shared_last += h_ctrl_[ph].shared_last;
            const bool grew = rows_out != nfront || frontier == nullptr;
            frontier = d_frontier_[buf];
            nfront = rows_out;
            last_frontier_rows_ = std::max(last_frontier_rows_, nfront);
            buf ^= 1;
            cur = nfront;
            if (!grew) break;
        }
    }
    EnumParams D = P;
    D.mode = rows ? CSM_ENUM_MODE_ROWS : CSM_ENUM_MODE_COUNT;
    // Work donation in the depth-first launch for every strategy but 1 ("DFS w/o work
    // stealing"); after a BFS phase (strategy 3) it evens out the frontier items' subtrees.
    D.donate = strategy == 1 ? 0u : 1u;
    if (frontier) {
        D.frontier = frontier;
        launch_ctrl_reset(sc_.ctrl, 0, nfront, s);
        stats_.kernel_launches++;
    }
    if (!rows && !memo_plan_.empty()) {
        // Tables of the pendant plans for this phase's graph and flags.
        for (size_t t = 0; t < memo_plan_.size(); t++)
            launch_pendant_counts(D, memo_plan_[t], d_memo_ + t * (size_t)g_.V, s);
        stats_.kernel_launches += memo_plan_.size();
        D.memo = d_memo_;
    }
    launch_enumerate(D, blocks_, warps_per_block_, occupancy_, s);
    stats_.enum_launches++;
    stats_.kernel_launches++;
    CSM_CUDA(record_event(ev_[3 + 2 * ph], s));
    // Statistics and error bits are read after the batch's final synchronisation.
    CSM_CUDA(cudaMemcpyAsync(&h_ctrl_[ph], sc_.ctrl, sizeof(EnumControl), cudaMemcpyDeviceToHost, s));
    if (rows) {
        // Collect rows per query for csm_get_embeddings (a validation path: synchronous).
        CSM_CUDA(cudaStreamSynchronize(s));
        const EnumControl &c = h_ctrl_[ph];
        if (c.error & (CSM_ERRBIT_OUTPUT | CSM_ERRBIT_TIMEOUT)) return CSM_OK;  // reported by run_batch
        const unsigned long long nr = c.out_rows;
        std::vector<uint32_t> h(nr * CSM_ROW_WORDS);
        if (nr) CSM_CUDA(cudaMemcpy(h.data(), d_rows_, sizeof(uint32_t) * h.size(), cudaMemcpyDeviceToHost));
        auto &dst = last_rows_[phase == CSM_PHASE_INS ? 0 : 1];
        dst.assign(queries_.size(), {});
        for (unsigned long long r = 0; r < nr; r++) {
            const uint32_t *row = &h[r * CSM_ROW_WORDS];
            const uint32_t qi = row[0];
            dst[qi].insert(dst[qi].end(), row + 1, row + 1 + queries_[qi].nv);
        }
    }
    return CSM_OK;
}

csm_status Engine::maybe_compact(cudaStream_t s) {
    const unsigned long long used = stats_.pool_used;
    const uint64_t max_batch = batch_cap_ ? batch_cap_ : 65536;
    const unsigned long long headroom = 64ull * max_batch + (1u << 20);
    if (used + headroom < g_.pool_cap && used < g_.pool_cap / 4 * 3) return CSM_OK;
    // Lay every list out again with fresh slack, growing the pool when the live lists leave too
    // little room.  The layout is computed first; the graph changes only once a pool for it has
    // been allocated, so a failure here leaves the current layout intact.
    unsigned long long *offsets = nullptr, total = 0;
    cudaError_t e = store_layout(g_, &offsets, total, s);
    if (e != cudaSuccess) return cuda_fail(e, "pool compaction layout");
    const unsigned long long limit = 0xFFFFFFF0ull;
    auto roomy = [&](unsigned long long cap) { return total + headroom < cap && total < cap / 4 * 3; };
    unsigned long long want = g_.pool_cap;
    if (!roomy(want)) want = std::min(limit, std::max(want * 2, 2 * (total + headroom)));
    uint32_t *np = nullptr;
    e = total <= want ? dev_alloc(&np, want) : cudaErrorMemoryAllocation;
    if (e == cudaErrorMemoryAllocation && want > g_.pool_cap && total <= g_.pool_cap) {
        // No memory to grow: a same-size pool still recovers the slack of relocated lists.
        cudaGetLastError();
        want = g_.pool_cap;
        e = dev_alloc(&np, want);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(offsets);
        return fail(CSM_ERR_OOM, "adjacency pool cannot be compacted: the live lists need " + std::to_string(total) +
                                     " entries");
    }
    e = store_relayout(g_, np, offsets, total, s);
    cudaFree(offsets);
    if (e != cudaSuccess) {
        cudaFree(np);
        poisoned_ = true;
        return cuda_fail(e, "pool compaction");
    }
    cudaFree(g_.pool);
    g_.pool = np;
    g_.pool_cap = want;
    clear_graphs();
    graph_gen_++;
    stats_.pool_used = total;
    stats_.pool_capacity = want;
    stats_.compactions++;
    return CSM_OK;
}

csm_status Engine::edge_counts(int32_t qid, uint64_t *pos, uint64_t *neg, uint32_t capacity, uint32_t *n_out) const {
    if (qid < 0 || qid >= (int32_t)queries_.size()) return CSM_ERR_INVALID_ARG;
    if (!graph_loaded_) return CSM_ERR_STATE;
    const uint32_t np = (uint32_t)plans_.size();
    const uint32_t b = plan_begin_[qid], e = plan_begin_[qid + 1];
    if (n_out) *n_out = e - b;
    for (uint32_t p = b; p < e && p - b < capacity; p++) {
        if (pos) pos[p - b] = last_counts_[p + np];
        if (neg) neg[p - b] = last_counts_[p];
    }
    return CSM_OK;
}

csm_status Engine::embeddings(int32_t qid, int32_t sign, uint32_t **rows, uint64_t *nrows) {
    if (qid < 0 || qid >= (int32_t)queries_.size() || !rows || !nrows)
        return fail(CSM_ERR_INVALID_ARG, "bad embeddings arguments");
    if (!cfg_.materialize_rows) return fail(CSM_ERR_STATE, "rows are kept only with materialize_rows > 0");
    if (!rows_valid_) return fail(CSM_ERR_STATE, "no batch has been applied");
    const auto &src = last_rows_[sign >= 0 ? 0 : 1];
    const uint32_t nv = queries_[qid].nv;
    std::vector<uint32_t> flat = qid < (int32_t)src.size() ? src[qid] : std::vector<uint32_t>();
    const uint64_t nr = flat.size() / nv;
    std::vector<uint64_t> idx(nr);
    for (uint64_t i = 0; i < nr; i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
        return std::lexicographical_compare(flat.begin() + a * nv, flat.begin() + (a + 1) * nv, flat.begin() + b * nv,
                                            flat.begin() + (b + 1) * nv);
    });
    uint32_t *outp = (uint32_t *)malloc(sizeof(uint32_t) * (nr * nv + 1));
    if (!outp) return fail(CSM_ERR_OOM, "host allocation for rows");
    for (uint64_t i = 0; i < nr; i++) std::memcpy(outp + i * nv, flat.data() + idx[i] * nv, sizeof(uint32_t) * nv);
    *rows = outp;
    *nrows = nr;
    return CSM_OK;
}

csm_status Engine::describe(int32_t qid, char *buf, size_t n) const {
    if (qid < 0 || qid >= (int32_t)queries_.size() || !buf || n == 0) return CSM_ERR_INVALID_ARG;
    if (!graph_loaded_) return CSM_ERR_STATE;
    std::vector<HostPlan> ps(plans_.begin() + plan_begin_[qid], plans_.begin() + plan_begin_[qid + 1]);
    std::string s = describe_plans(queries_[qid], ps);
    std::snprintf(buf, n, "%s", s.c_str());
    return CSM_OK;
}

csm_status Engine::stats(csm_stats *out) const {
    if (!out) return CSM_ERR_INVALID_ARG;
    *out = stats_;
    return CSM_OK;
}

void Engine::reset_stats() {
    const uint64_t used = stats_.pool_used, cap = stats_.pool_capacity;
    std::memset(&stats_, 0, sizeof(stats_));
    stats_.pool_used = used;
    stats_.pool_capacity = cap;
    // The launch configuration in use is state, not a counter.
    stats_.tuned_strategy = (uint64_t)lc_.strategy;
    stats_.tuned_steal_chunk = lc_.steal_chunk;
    stats_.tuned_warps_per_block = (uint64_t)lc_.warps_per_block;
    stats_.tuned_occupancy = (uint64_t)lc_.occupancy;
}

csm_status Engine::memory(uint64_t *free_b, uint64_t *total_b) const {
    size_t f = 0, t = 0;
    cudaError_t e = cudaMemGetInfo(&f, &t);
    if (e != cudaSuccess) return CSM_ERR_CUDA;
    if (free_b) *free_b = f;
    if (total_b) *total_b = t;
    return CSM_OK;
}

}  // namespace csm
