// csm_apply_batch_device_static: the batch pipeline for callers that must not allocate.
//
// Some callers cannot call cudaMalloc while they apply updates: serving processes that reserve
// their whole device-memory budget up front and forbid allocation afterwards (to avoid
// fragmentation and the device-wide synchronisation that cudaMalloc/cudaFree can imply),
// and hosts that embed this engine as a plugin inside a runtime that owns all device memory.
// This entry point runs the same pipeline as csm_apply_batch_device, but the scratch of the
// enumeration kernel (its control block, the work-donation queue with its ready flags, and the
// per-plan seed ranges and ticket prefixes) lives in one fixed array compiled into the library,
// and nothing is allocated or regrown during the call.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine_handle.h"

namespace {

constexpr size_t kScratchBytes = CSM_STATIC_SCRATCH_BYTES;
constexpr uint32_t kMaxPlans = CSM_STATIC_MAX_PLANS;

// The scratch array.  Every GPU that loads the library holds it until the process exits.
// In host code `g_scratch` only names the symbol: its device address comes from
// cudaGetSymbolAddress, resolved once per device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kCtrlOff = 0;
constexpr size_t kSeedOff = align256(sizeof(EnumControl));
constexpr size_t kTicketOff = kSeedOff + align256(sizeof(uint32_t) * 3 * kMaxPlans);
constexpr size_t kReadyOff = kTicketOff + align256(sizeof(uint32_t) * (kMaxPlans + 1));
constexpr uint32_t kQueueItems =
    (uint32_t)((kScratchBytes - kReadyOff - 256) / (sizeof(uint32_t) + sizeof(WorkItem)));
constexpr size_t kQueueOff = align256(kReadyOff + sizeof(uint32_t) * kQueueItems);
static_assert(kQueueOff + sizeof(WorkItem) * kQueueItems <= kScratchBytes, "scratch layout overflows");

std::mutex g_mutex;
constexpr int kMaxDevices = 128;
void *g_device_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
cudaError_t scratch_address(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_device_ptr[device]) {
        void *p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_scratch);
        if (rc != cudaSuccess) return rc;
        g_device_ptr[device] = p;
    }
    *out = g_device_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" csm_status csm_apply_batch_device_static(csm_engine *e, uint64_t n, const uint32_t *d_src,
                                                    const uint32_t *d_dst, const uint32_t *d_elabel,
                                                    const uint8_t *d_is_delete, void *stream,
                                                    csm_batch_result *per_query_out) {
    if (!e) return CSM_ERR_INVALID_ARG;
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
    const cudaError_t rc = scratch_address(dev, &base);
    if (rc != cudaSuccess) {
        st = eng.fail(CSM_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(rc));
    } else {
        unsigned char *b = static_cast<unsigned char *>(base);
        csm::EnumScratch sc;
        sc.ctrl = reinterpret_cast<EnumControl *>(b + kCtrlOff);
        sc.seed_lo = reinterpret_cast<uint32_t *>(b + kSeedOff);
        sc.ticket_prefix = reinterpret_cast<uint32_t *>(b + kTicketOff);
        sc.ready = reinterpret_cast<uint32_t *>(b + kReadyOff);
        sc.queue = reinterpret_cast<WorkItem *>(b + kQueueOff);
        sc.qcap = kQueueItems;
        // The array keeps the previous call's contents: the ready flags of the donation queue
        // must start at zero (the control block is reset before every launch).
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : eng.stream();
        const cudaError_t mc = cudaMemsetAsync(sc.ready, 0, sizeof(uint32_t) * kQueueItems, s);
        if (mc != cudaSuccess)
            st = eng.fail(CSM_ERR_CUDA, std::string("clearing the static scratch: ") + cudaGetErrorString(mc));
        else
            st = eng.apply_device_noalloc(n, d_src, d_dst, d_elabel, d_is_delete, s, sc, per_query_out);
    }
    if (prev != dev) cudaSetDevice(prev);
    return st;
}
