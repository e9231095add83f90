// Continuous-batching serving loop over engines on one GPU (include/csm_server.h).
//
// Slots are worker threads, each with a non-blocking CUDA stream, its own enumeration scratch
// (control block, donation queue and ready flags, seed arrays) and a pinned staging buffer for
// the update arrays.  A slot takes the oldest admissible work unit (one request on one tenant),
// borrows a frontier from the arena and runs the tenant engine's batch pipeline on its stream;
// units of different tenants therefore overlap on the device.  The reference's driver
// (technique_permutation.h:121-214) runs one batch at a time on the default stream; nothing in
// it corresponds to this file.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/csm_server.h"
#include "engine_handle.h"
#include "frontier_arena.h"

namespace csm {
namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

constexpr uint32_t kSlotQueueItems = 1u << 18;  // donation ring slots per slot (reused)
constexpr uint32_t kSlotMaxPlans = 4096;

// The device range behind the frontier arena (bookkeeping in RangeAllocator).
class FrontierArena {
  public:
    cudaError_t init(uint64_t bytes) {
        ra_.reset(bytes);
        if (!ra_.size()) return cudaSuccess;
        cudaError_t e = cudaMalloc(&base_, ra_.size());
        if (e != cudaSuccess) ra_.reset(0);
        return e;
    }
    void release() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
        ra_.reset(0);
    }
    uint64_t take(uint64_t want, uint64_t least, char **ptr) {
        uint64_t off = 0;
        const uint64_t got = ra_.take(want, least, &off);
        if (got) *ptr = base_ + off;
        return got;
    }
    void give(char *ptr, uint64_t bytes) {
        if (bytes) ra_.give((uint64_t)(ptr - base_), bytes);
    }
    uint64_t used() const { return ra_.used(); }
    uint64_t size() const { return ra_.size(); }

  private:
    char *base_ = nullptr;
    RangeAllocator ra_;
};

struct Request {
    uint64_t id = 0;
    int32_t tenant = -1;
    std::vector<uint32_t> src, dst, lab;
    std::vector<uint8_t> del;
    bool has_delete = false;
    uint32_t units_left = 0;
    std::vector<uint32_t> result_offset;  // per tenant: first result index (broadcast requests)
    std::vector<csm_batch_result> results;
    csm_request_info info{};
    bool done = false;
};

struct Tenant {
    Engine *eng = nullptr;
    bool busy = false;
    std::deque<Request *> pending;
    double rows_per_update = 0.0;  // recent semi-BFS frontier items per update (running average)
};

struct Slot {
    cudaStream_t stream = nullptr;
    EnumScratch sc;
    char *pinned = nullptr;
    uint64_t pinned_bytes = 0;
    std::thread th;
};

}  // namespace

class Server {
  public:
    explicit Server(const csm_server_config &c) : cfg_(c) {}
    ~Server() { shutdown(); }

    csm_status init() {
        if (cfg_.slots <= 0) cfg_.slots = 4;
        if (cfg_.slots > 64) return fail(CSM_ERR_INVALID_ARG, "at most 64 slots");
        if (!cfg_.memory_budget) cfg_.memory_budget = 8ull << 30;
        if (!cfg_.min_frontier_bytes) cfg_.min_frontier_bytes = 16ull << 20;
        if (!cfg_.max_pending) cfg_.max_pending = 4096;
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CSM_ERR_NO_DEVICE, "no CUDA device");
        if (cfg_.device < 0 || cfg_.device >= ndev) return fail(CSM_ERR_INVALID_ARG, "device out of range");
        cudaError_t e = cudaSetDevice(cfg_.device);
        if (e == cudaSuccess) e = arena_.init(cfg_.memory_budget);
        if (e != cudaSuccess) return cuda_fail(e, "frontier arena");
        slots_.resize((size_t)cfg_.slots);
        for (auto &sl : slots_) {
            e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaMalloc(&sl.sc.ctrl, sizeof(EnumControl));
            if (e == cudaSuccess) e = cudaMemset(sl.sc.ctrl, 0, sizeof(EnumControl));
            if (e == cudaSuccess) e = cudaMalloc(&sl.sc.queue, sizeof(WorkItem) * kSlotQueueItems);
            if (e == cudaSuccess) e = cudaMalloc(&sl.sc.seq, sizeof(unsigned long long) * kSlotQueueItems);
            if (e == cudaSuccess) e = cudaMemset(sl.sc.seq, 0, sizeof(unsigned long long) * kSlotQueueItems);
            if (e == cudaSuccess) e = cudaMalloc(&sl.sc.seed_lo, sizeof(uint32_t) * 3 * kSlotMaxPlans);
            if (e == cudaSuccess) e = cudaMalloc(&sl.sc.ticket_prefix, sizeof(uint32_t) * (kSlotMaxPlans + 1));
            if (e != cudaSuccess) return cuda_fail(e, "slot scratch");
            sl.sc.qcap = kSlotQueueItems;
        }
        for (size_t i = 0; i < slots_.size(); i++) slots_[i].th = std::thread([this, i] { worker(i); });
        started_ = true;
        return CSM_OK;
    }

    csm_status add_tenant(Engine *eng, int32_t *out) {
        if (!eng || !out) return fail(CSM_ERR_INVALID_ARG, "null argument");
        std::lock_guard<std::mutex> lk(mu_);
        if (eng->device() != cfg_.device) return fail(CSM_ERR_INVALID_ARG, "engine is on another device");
        if (!eng->graph_loaded()) return fail(CSM_ERR_STATE, "load the engine's queries and graph first");
        if (eng->num_plans() > kSlotMaxPlans) return fail(CSM_ERR_LIMIT, "engine has more than 4096 query edges");
        for (auto &t : tenants_)
            if (t.eng == eng) return fail(CSM_ERR_INVALID_ARG, "engine already added");
        if (!reqs_.empty()) return fail(CSM_ERR_STATE, "add tenants before the first request");
        tenants_.emplace_back();
        tenants_.back().eng = eng;
        *out = (int32_t)tenants_.size() - 1;
        return CSM_OK;
    }

    csm_status submit(int32_t tenant, uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *lab,
                      const uint8_t *del, uint64_t *out) {
        if (!out) return fail(CSM_ERR_INVALID_ARG, "null request id");
        if (n && (!src || !dst || !lab)) return fail(CSM_ERR_INVALID_ARG, "null update array");
        auto r = std::make_unique<Request>();
        r->src.assign(src, src + n);
        r->dst.assign(dst, dst + n);
        r->lab.assign(lab, lab + n);
        if (del) {
            r->del.assign(del, del + n);
            r->has_delete = std::any_of(r->del.begin(), r->del.end(), [](uint8_t x) { return x != 0; });
        }
        std::lock_guard<std::mutex> lk(mu_);
        if (stopping_) return fail(CSM_ERR_STATE, "server is shutting down");
        if (tenants_.empty()) return fail(CSM_ERR_STATE, "no tenants");
        if (tenant < -1 || tenant >= (int32_t)tenants_.size()) return fail(CSM_ERR_INVALID_ARG, "no such tenant");
        if (reqs_.size() >= cfg_.max_pending) return fail(CSM_ERR_LIMIT, "too many requests not yet waited for");
        r->id = ++next_id_;
        r->tenant = tenant;
        r->info.arrival_ns = now_ns();
        r->info.frontier_bytes = ~0ull;
        const size_t t0 = tenant < 0 ? 0 : (size_t)tenant;
        const size_t t1 = tenant < 0 ? tenants_.size() : (size_t)tenant + 1;
        r->result_offset.assign(tenants_.size(), 0);
        uint32_t nres = 0;
        for (size_t t = t0; t < t1; t++) {
            r->result_offset[t] = nres;
            nres += tenants_[t].eng->num_queries();
        }
        r->results.assign(nres, csm_batch_result{});
        r->info.nresults = nres;
        r->units_left = (uint32_t)(t1 - t0);
        Request *rp = r.get();
        reqs_[r->id] = std::move(r);
        for (size_t t = t0; t < t1; t++) tenants_[t].pending.push_back(rp);
        *out = rp->id;
        work_cv_.notify_all();
        return CSM_OK;
    }

    csm_status wait(uint64_t id, int64_t timeout_ms, csm_request_info *info, csm_batch_result *res, uint32_t cap) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) return fail(CSM_ERR_INVALID_ARG, "unknown request (or already waited for)");
        Request *r = it->second.get();
        auto ready = [r] { return r->done; };
        if (timeout_ms < 0)
            done_cv_.wait(lk, ready);
        else if (!done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return CSM_ERR_TIMEOUT;
        if (info) *info = r->info;
        if (res) std::memcpy(res, r->results.data(), sizeof(csm_batch_result) * std::min<size_t>(cap, r->results.size()));
        const csm_status st = r->info.status;
        if (st != CSM_OK) fail(st, r_err_[id]);
        r_err_.erase(id);
        reqs_.erase(it);
        return st;
    }

    void stats(csm_server_stats *out) const {
        std::lock_guard<std::mutex> lk(mu_);
        *out = stats_;
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stopping_ = true;
        }
        work_cv_.notify_all();
        for (auto &sl : slots_)
            if (sl.th.joinable()) sl.th.join();
        if (!started_ && slots_.empty()) return;
        cudaSetDevice(cfg_.device);
        for (auto &sl : slots_) {
            if (sl.stream) cudaStreamSynchronize(sl.stream);
            cudaFree(sl.sc.ctrl);
            cudaFree(sl.sc.queue);
            cudaFree(sl.sc.seq);
            cudaFree(sl.sc.seed_lo);
            cudaFree(sl.sc.ticket_prefix);
            if (sl.pinned) cudaFreeHost(sl.pinned);
            if (sl.stream) cudaStreamDestroy(sl.stream);
        }
        slots_.clear();
        arena_.release();
        started_ = false;
    }

    // The last error message (callers may ask from any thread).
    std::string error() const {
        std::lock_guard<std::mutex> g(err_mu_);
        return err_;
    }
    csm_status fail(csm_status code, const std::string &msg) {
        std::lock_guard<std::mutex> g(err_mu_);
        err_ = msg;
        return code;
    }
    csm_status cuda_fail(cudaError_t e, const char *where) {
        return fail(e == cudaErrorMemoryAllocation ? CSM_ERR_OOM : CSM_ERR_CUDA,
                    std::string(where) + ": " + cudaGetErrorString(e));
    }

  private:
    // Frontier bytes a unit asks for: two buffers of twice the items the tenant's semi-BFS
    // wrote per update recently, scaled to this batch, and at least twice the item count at
    // which the dynamic semi-BFS switches to depth first.  Depth-first tenants need none.
    uint64_t estimate(const Tenant &t, uint64_t n) const {
        if (t.eng->strategy() < 2) return 0;
        const double floor_items = 2.0 * (double)t.eng->semi_bfs_target_items();
        const double items = std::max(floor_items, 2.0 * t.rows_per_update * (double)n);
        const double bytes = 2.0 * items * (double)sizeof(WorkItem);
        return (uint64_t)std::min(bytes, (double)arena_.size());
    }

    // Picks the next unit (under the lock): the oldest runnable unit whose memory is granted,
    // or one that needs none.  Returns the tenant index or -1.
    int pick(char **fptr, uint64_t *grant) {
        std::vector<int> order;
        for (size_t t = 0; t < tenants_.size(); t++)
            if (!tenants_[t].busy && !tenants_[t].pending.empty()) order.push_back((int)t);
        std::sort(order.begin(), order.end(), [this](int a, int b) {
            return tenants_[a].pending.front()->id < tenants_[b].pending.front()->id;
        });
        bool blocked = false;
        for (int t : order) {
            Tenant &tn = tenants_[t];
            const uint64_t want = estimate(tn, tn.pending.front()->src.size());
            *fptr = nullptr;
            *grant = 0;
            if (want == 0) return t;
            if (blocked) continue;  // memory goes to the oldest unit first
            const uint64_t least = std::min<uint64_t>(want, cfg_.min_frontier_bytes);
            *grant = arena_.take(want, least, fptr);
            if (*grant) {
                if (*grant < want) stats_.units_shrunk++;
                return t;
            }
            if (arena_.used() == 0) return t;  // no unit holds memory to free: run depth first
            if (!mem_wait_counted_) {
                stats_.memory_waits++;
                mem_wait_counted_ = true;
            }
            blocked = true;
        }
        return -1;
    }

    void worker(size_t si) {
        Slot &sl = slots_[si];
        cudaSetDevice(cfg_.device);
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            char *fptr = nullptr;
            uint64_t grant = 0;
            int t = pick(&fptr, &grant);
            if (t < 0) {
                if (stopping_ && inflight_ == 0 && all_idle()) break;
                work_cv_.wait(lk);
                continue;
            }
            mem_wait_counted_ = false;
            Tenant &tn = tenants_[(size_t)t];
            Request *r = tn.pending.front();
            tn.pending.pop_front();
            tn.busy = true;
            inflight_++;
            stats_.peak_inflight = std::max<uint64_t>(stats_.peak_inflight, inflight_);
            stats_.peak_frontier_bytes = std::max(stats_.peak_frontier_bytes, arena_.used());
            if (!grant) stats_.units_depth_first++;
            if (!r->info.start_ns) r->info.start_ns = now_ns();
            r->info.frontier_bytes = std::min(r->info.frontier_bytes, grant);
            csm_batch_result *out = r->results.data() + r->result_offset[(size_t)t];
            lk.unlock();

            std::string uerr;
            const csm_status st = run_unit(sl, *tn.eng, *r, fptr, grant, out, &uerr);
            const unsigned long long rows = tn.eng->last_frontier_rows();

            lk.lock();
            arena_.give(fptr, grant);
            const uint64_t n = r->src.size();
            if (st == CSM_OK && n) {
                const double rate = (double)rows / (double)n;
                tn.rows_per_update = tn.rows_per_update > 0 ? 0.5 * tn.rows_per_update + 0.5 * rate : rate;
            }
            tn.busy = false;
            inflight_--;
            stats_.units++;
            if (st == CSM_OK && n) r->info.device_ns += out[0].latency_ns;
            if (st != CSM_OK && r->info.status == CSM_OK) {
                r->info.status = st;
                r_err_[r->id] = uerr;
            }
            if (--r->units_left == 0) {
                r->info.done_ns = now_ns();
                if (r->info.frontier_bytes == ~0ull) r->info.frontier_bytes = 0;
                r->done = true;
                stats_.requests++;
                done_cv_.notify_all();
            }
            work_cv_.notify_all();
        }
    }

    bool all_idle() const {
        for (auto &t : tenants_)
            if (!t.pending.empty() || t.busy) return false;
        return true;
    }

    csm_status run_unit(Slot &sl, Engine &eng, const Request &r, char *fptr, uint64_t grant, csm_batch_result *out,
                        std::string *err) {
        const uint64_t n = r.src.size();
        const uint64_t need = 13 * n + 64;
        if (need > sl.pinned_bytes) {
            if (sl.pinned) cudaFreeHost(sl.pinned);
            sl.pinned = nullptr;
            sl.pinned_bytes = 0;
            cudaError_t e = cudaMallocHost(&sl.pinned, need * 2);
            if (e != cudaSuccess) {
                *err = std::string("pinned staging: ") + cudaGetErrorString(e);
                return CSM_ERR_OOM;
            }
            sl.pinned_bytes = need * 2;
        }
        uint32_t *ps = reinterpret_cast<uint32_t *>(sl.pinned);
        uint32_t *pd = ps + n, *pl = pd + n;
        uint8_t *pdel = reinterpret_cast<uint8_t *>(pl + n);
        if (n) {
            std::memcpy(ps, r.src.data(), 4 * n);
            std::memcpy(pd, r.dst.data(), 4 * n);
            std::memcpy(pl, r.lab.data(), 4 * n);
            if (r.has_delete) std::memcpy(pdel, r.del.data(), n);
        }
        ExecContext ctx;
        ctx.scratch = sl.sc;
        ctx.stream = sl.stream;
        const uint64_t half = grant / 2 / kGranule * kGranule;
        ctx.frontier_cap = half / sizeof(WorkItem);
        if (ctx.frontier_cap) {
            ctx.frontier[0] = reinterpret_cast<WorkItem *>(fptr);
            ctx.frontier[1] = reinterpret_cast<WorkItem *>(fptr + half);
        }
        const csm_status st = eng.apply_host_ctx(ctx, n, ps, pd, pl, r.has_delete ? pdel : nullptr, out);
        if (st != CSM_OK) *err = eng.error();
        return st;
    }

    csm_server_config cfg_;
    mutable std::mutex mu_;
    std::condition_variable work_cv_, done_cv_;
    std::deque<Tenant> tenants_;  // stable references while units run
    std::vector<Slot> slots_;
    std::map<uint64_t, std::unique_ptr<Request>> reqs_;
    std::map<uint64_t, std::string> r_err_;
    FrontierArena arena_;
    csm_server_stats stats_{};
    uint64_t next_id_ = 0;
    uint32_t inflight_ = 0;
    bool stopping_ = false, started_ = false, mem_wait_counted_ = false;
    mutable std::mutex err_mu_;
    std::string err_;
};

}  // namespace csm

struct csm_server {
    csm::Server impl;
    explicit csm_server(const csm_server_config &c) : impl(c) {}
};

namespace {
thread_local std::string g_server_create_error;
}

extern "C" {

csm_status csm_server_default_config(csm_server_config *cfg) {
    if (!cfg) return CSM_ERR_INVALID_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->slots = 4;
    cfg->memory_budget = 8ull << 30;
    cfg->min_frontier_bytes = 16ull << 20;
    cfg->max_pending = 4096;
    return CSM_OK;
}

csm_status csm_server_create(csm_server **out, const csm_server_config *cfg) {
    if (!out) return CSM_ERR_INVALID_ARG;
    *out = nullptr;
    csm_server_config c;
    if (cfg)
        c = *cfg;
    else
        csm_server_default_config(&c);
    csm_server *s = new (std::nothrow) csm_server(c);
    if (!s) return CSM_ERR_OOM;
    csm_status st = s->impl.init();
    if (st != CSM_OK) {
        g_server_create_error = s->impl.error();
        delete s;
        return st;
    }
    *out = s;
    return CSM_OK;
}

csm_status csm_server_add_tenant(csm_server *srv, csm_engine *engine, int32_t *tenant_out) {
    if (!srv || !engine) return CSM_ERR_INVALID_ARG;
    return srv->impl.add_tenant(&engine->impl, tenant_out);
}

csm_status csm_server_submit(csm_server *srv, int32_t tenant, uint64_t n, const uint32_t *src, const uint32_t *dst,
                             const uint32_t *elabel, const uint8_t *is_delete, uint64_t *request_out) {
    if (!srv) return CSM_ERR_INVALID_ARG;
    try {
        return srv->impl.submit(tenant, n, src, dst, elabel, is_delete, request_out);
    } catch (const std::bad_alloc &) {
        return srv->impl.fail(CSM_ERR_OOM, "host allocation failed");
    }
}

csm_status csm_server_wait(csm_server *srv, uint64_t request, int64_t timeout_ms, csm_request_info *info,
                           csm_batch_result *results, uint32_t capacity) {
    if (!srv) return CSM_ERR_INVALID_ARG;
    return srv->impl.wait(request, timeout_ms, info, results, capacity);
}

csm_status csm_server_get_stats(const csm_server *srv, csm_server_stats *out) {
    if (!srv || !out) return CSM_ERR_INVALID_ARG;
    srv->impl.stats(out);
    return CSM_OK;
}

csm_status csm_server_destroy(csm_server *srv) {
    if (!srv) return CSM_ERR_INVALID_ARG;
    srv->impl.shutdown();
    delete srv;
    return CSM_OK;
}

csm_status csm_server_last_error(const csm_server *srv, char *buf, size_t n) {
    if (!buf || !n) return CSM_ERR_INVALID_ARG;
    const std::string s = srv ? srv->impl.error() : g_server_create_error;
    const size_t k = std::min(n - 1, s.size());
    std::memcpy(buf, s.data(), k);
    buf[k] = 0;
    return CSM_OK;
}

}  // extern "C"
