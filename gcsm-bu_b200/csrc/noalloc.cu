// csm_apply_batch_device_static: the batch pipeline for callers that must not allocate.
//
// Some callers cannot call cudaMalloc while they apply updates: serving processes that reserve
// their whole device-memory budget up front and forbid allocation afterwards (to avoid
// fragmentation and the device-wide synchronisation that cudaMalloc/cudaFree can imply),
// and hosts that embed this engine as a plugin inside a runtime that owns all device memory.
// This entry point runs the same pipeline as csm_apply_batch_device, but the scratch of the
// enumeration kernel (its control block, the work-donation ring with its sequence words, and
// the per-plan seed ranges and ticket prefixes) lives in one fixed array compiled into the
// library, and nothing is allocated or regrown during the call.
#include <cuda_runtime.h>

#include <new>
#include <string>

#include "engine_handle.h"

namespace {

constexpr size_t kScratchBytes = CSM_STATIC_SCRATCH_BYTES;
constexpr uint32_t kMaxPlans = CSM_STATIC_MAX_PLANS;

// The scratch array.  Every GPU that loads the library holds it until the process exits.
// In host code `g_scratch` only names the symbol: its device address comes from
// cudaGetSymbolAddress (Engine::static_scratch, once per engine, with its device current).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kCtrlOff = 0;
constexpr size_t kSeedOff = align256(sizeof(EnumControl));
constexpr size_t kTicketOff = kSeedOff + align256(sizeof(uint32_t) * 3 * kMaxPlans);
constexpr size_t kSeqOff = kTicketOff + align256(sizeof(uint32_t) * (kMaxPlans + 1));
// Ring slots: the largest power of two whose sequence words and items fit the rest.
constexpr uint32_t ring_slots() {
    uint32_t q = 1u << 30;
    while (q > CSM_QUEUE_MIN_SLOTS &&
           align256(kSeqOff + sizeof(unsigned long long) * q) + sizeof(WorkItem) * (size_t)q > kScratchBytes)
        q >>= 1;
    return q;
}
constexpr uint32_t kQueueItems = ring_slots();
constexpr size_t kQueueOff = align256(kSeqOff + sizeof(unsigned long long) * kQueueItems);
static_assert(kQueueOff + sizeof(WorkItem) * kQueueItems <= kScratchBytes, "scratch layout overflows");
static_assert(kQueueItems >= 4096, "the static donation ring is too small to balance a launch");

cudaError_t lookup_scratch(void **out) { return cudaGetSymbolAddress(out, g_scratch); }

csm_status apply_static(csm_engine *e, uint64_t n, const uint32_t *d_src, const uint32_t *d_dst,
                        const uint32_t *d_elabel, const uint8_t *d_is_delete, void *stream,
                        csm_batch_result *per_query_out) {
    csm::Engine &eng = e->impl;
    if (eng.num_plans() > kMaxPlans)
        return eng.fail(CSM_ERR_LIMIT, "the registered queries have " + std::to_string(eng.num_plans()) +
                                           " query edges in total; the static scratch holds at most " +
                                           std::to_string(kMaxPlans));
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return eng.fail(CSM_ERR_CUDA, "cudaGetDevice failed");
    const int dev = eng.device();
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return eng.fail(CSM_ERR_CUDA, "cudaSetDevice failed");
    csm_status st = CSM_OK;
    void *base = nullptr;
    const cudaError_t rc = eng.static_scratch(lookup_scratch, &base);
    if (rc != cudaSuccess) {
        st = eng.fail(CSM_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(rc));
    } else {
        unsigned char *b = static_cast<unsigned char *>(base);
        csm::EnumScratch sc;
        sc.ctrl = reinterpret_cast<EnumControl *>(b + kCtrlOff);
        sc.seed_lo = reinterpret_cast<uint32_t *>(b + kSeedOff);
        sc.ticket_prefix = reinterpret_cast<uint32_t *>(b + kTicketOff);
        sc.seq = reinterpret_cast<unsigned long long *>(b + kSeqOff);
        sc.queue = reinterpret_cast<WorkItem *>(b + kQueueOff);
        sc.qcap = kQueueItems;
        // The array keeps the previous call's contents, and nothing in it has to be cleared:
        // the control block is rewritten before every launch, and the ring's sequence words
        // carry the launch epoch, so words left by earlier calls never read as fresh.
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : eng.stream();
        st = eng.apply_device_noalloc(n, d_src, d_dst, d_elabel, d_is_delete, s, sc, per_query_out);
    }
    if (prev != dev) cudaSetDevice(prev);
    return st;
}

}  // namespace

extern "C" csm_status csm_apply_batch_device_static(csm_engine *e, uint64_t n, const uint32_t *d_src,
                                                    const uint32_t *d_dst, const uint32_t *d_elabel,
                                                    const uint8_t *d_is_delete, void *stream,
                                                    csm_batch_result *per_query_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
    // No exception may leave an extern "C" function (it would end the process).
    try {
        return apply_static(e, n, d_src, d_dst, d_elabel, d_is_delete, stream, per_query_out);
    } catch (const std::bad_alloc &) {
        e->impl.fail(CSM_ERR_OOM, "host allocation failed");
        return CSM_ERR_OOM;
    } catch (const std::exception &ex) {
        e->impl.fail(CSM_ERR_STATE, ex.what());
        return CSM_ERR_STATE;
    }
}
