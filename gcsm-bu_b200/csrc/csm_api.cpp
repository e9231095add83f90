// extern "C" entry points of libcsm.so (declared in include/csm.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "engine_handle.h"

namespace {

thread_local std::string g_create_error;

template <typename F>
csm_status guarded(csm_engine *e, F &&f) {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        if (e) e->impl.fail(CSM_ERR_OOM, "host allocation failed");
        return CSM_ERR_OOM;
    } catch (const std::exception &ex) {
        if (e) e->impl.fail(CSM_ERR_STATE, ex.what());
        return CSM_ERR_STATE;
    }
}

}  // namespace

extern "C" {

const char *csm_version(void) { return "csm-b200 0.1 (sm_100a)"; }

csm_status csm_default_config(csm_config *cfg) {
    if (!cfg) return CSM_ERR_INVALID_ARG;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = 0;
    cfg->algorithm = 0;
    cfg->matching_order = 2;
    cfg->search_strategy = 2;
    cfg->local_index = 1;
    cfg->cartesian_product = 1;
    cfg->heavy_vertex_avoidance = 1;
    cfg->relation_switch = 1;
    return CSM_OK;
}

csm_status csm_create(csm_engine **out, const csm_config *cfg) {
    if (!out) return CSM_ERR_INVALID_ARG;
    *out = nullptr;
    csm_config c;
    if (cfg) c = *cfg;
    else csm_default_config(&c);
    csm_engine *e = nullptr;
    try {
        e = new csm_engine(c);
    } catch (...) {
        g_create_error = "host allocation failed";
        return CSM_ERR_OOM;
    }
    csm_status st = e->impl.init();
    if (st != CSM_OK) {
        g_create_error = e->impl.error();
        delete e;
        return st;
    }
    *out = e;
    return CSM_OK;
}

csm_status csm_destroy(csm_engine *e) {
    delete e;
    return CSM_OK;
}

csm_status csm_load_query(csm_engine *e, uint32_t nv, const uint32_t *vlabel, uint32_t ne, const uint32_t *src,
                          const uint32_t *dst, const uint32_t *elabel, int32_t *query_id_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] { return e->impl.load_query(nv, vlabel, ne, src, dst, elabel, query_id_out); });
}

csm_status csm_load_graph(csm_engine *e, uint32_t nv, const uint32_t *vlabel, uint64_t ne, const uint32_t *src,
                          const uint32_t *dst, const uint32_t *elabel) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] { return e->impl.load_graph(nv, vlabel, ne, src, dst, elabel); });
}

csm_status csm_save_snapshot(csm_engine *e, const char *path) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] { return e->impl.save_snapshot(path); });
}

csm_status csm_load_snapshot(csm_engine *e, const char *path) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] { return e->impl.load_snapshot(path); });
}

csm_status csm_apply_batch(csm_engine *e, uint64_t n, const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                           const uint8_t *is_delete, csm_batch_result *per_query_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] { return e->impl.apply_host(n, src, dst, elabel, is_delete, per_query_out); });
}

csm_status csm_apply_batch_device(csm_engine *e, uint64_t n, const uint32_t *d_src, const uint32_t *d_dst,
                                  const uint32_t *d_elabel, const uint8_t *d_is_delete, void *stream,
                                  csm_batch_result *per_query_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] {
        return e->impl.apply_device(n, d_src, d_dst, d_elabel, d_is_delete, (cudaStream_t)stream, per_query_out);
    });
}

csm_status csm_set_time_limit(csm_engine *e, uint64_t time_limit_us) {
    if (!e) return CSM_ERR_INVALID_ARG;
    e->impl.set_time_limit_us(time_limit_us);
    return CSM_OK;
}

csm_status csm_get_edge_counts(const csm_engine *e, int32_t query_id, uint64_t *positive, uint64_t *negative,
                               uint32_t capacity, uint32_t *n_edges_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return e->impl.edge_counts(query_id, positive, negative, capacity, n_edges_out);
}

csm_status csm_get_embeddings(csm_engine *e, int32_t query_id, int32_t sign, uint32_t **rows_out, uint64_t *nrows_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return guarded(e, [&] { return e->impl.embeddings(query_id, sign, rows_out, nrows_out); });
}

csm_status csm_free(void *ptr) {
    std::free(ptr);
    return CSM_OK;
}

csm_status csm_describe_plan(const csm_engine *e, int32_t query_id, char *buf, size_t n) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return e->impl.describe(query_id, buf, n);
}

csm_status csm_get_stats(const csm_engine *e, csm_stats *out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return e->impl.stats(out);
}

csm_status csm_reset_stats(csm_engine *e) {
    if (!e) return CSM_ERR_INVALID_ARG;
    e->impl.reset_stats();
    return CSM_OK;
}

csm_status csm_device_memory(const csm_engine *e, uint64_t *free_bytes, uint64_t *total_bytes) {
    if (!e) return CSM_ERR_INVALID_ARG;
    return e->impl.memory(free_bytes, total_bytes);
}

csm_status csm_last_error(const csm_engine *e, char *buf, size_t n) {
    if (!buf || n == 0) return CSM_ERR_INVALID_ARG;
    const std::string &s = e ? e->impl.error() : g_create_error;
    std::snprintf(buf, n, "%s", s.c_str());
    return CSM_OK;
}

}  // extern "C"
