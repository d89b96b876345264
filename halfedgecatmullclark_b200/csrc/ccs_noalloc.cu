// ccs_noalloc.cu -- the adjoint entry point that allocates no GPU memory.
//
// ccs_AdjointPointsDevice_cuda keeps a working buffer (one float triple per
// refined point) that it allocates with cudaMalloc the first time it runs.
// Callers that cannot let a library allocate -- a graph being recorded by
// stream capture, where cudaMalloc is not permitted; an application whose
// pool allocator owns the device memory; a real-time loop that forbids
// allocation after start-up -- call ccs_AdjointPointsDeviceNoAlloc_cuda
// instead.  Its working buffer is the fixed array below, part of the
// library image: every GPU that loads the library holds these 16 MiB until
// the process exits.
//
// The array is shared by every call in the process and keeps whatever the
// last call left in it.  The adjoint overwrites all of the part it uses
// (it starts by copying the incoming gradient into it), so nothing needs
// clearing; but two calls whose kernels overlap on the GPU race on it, and
// the caller must serialise them.
#include <mutex>

#include "ccs_host.h"

namespace ccs {

int adjoint_into(const cc_Subd* subd, const float* gradPoints, float* gradCage, float* work, int64_t workFloats,
                 cudaStream_t stream);
int set_last_error(int status);

// 16 MiB: the work buffer of subds with up to 1,398,101 refined points.
static constexpr int64_t kScratchFloats = 4 * 1024 * 1024;
static __device__ __align__(256) float g_adjoint_scratch[kScratchFloats];

// Host code must not use g_adjoint_scratch itself (on the host it names a
// host-side stand-in, not GPU memory): it uses the device address looked up
// with that device current, once per device and context.  The context's id
// is kept beside the address: a caller that resets the device
// (cudaDeviceReset) gets a new context, whose address is looked up again.
static constexpr int kMaxDevices = 64;
struct ScratchSlot {
    float* addr = nullptr;
    unsigned long long ctx = 0;
};
static std::mutex g_scratch_mu;
static ScratchSlot g_scratch[kMaxDevices];

// The unique id of the calling thread's current context (cuCtxGetId, through
// the runtime's driver entry points: no link against the driver library);
// false when it cannot be read, in which case nothing is cached.
static bool current_context_id(unsigned long long* id) {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
    });
    void* ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, id) == 0;
}

static int scratch_address(float** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CCS_ERR_CUDA;
    unsigned long long ctx = 0;
    const bool known = current_context_id(&ctx);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    ScratchSlot& slot = g_scratch[dev];
    if (!known || !slot.addr || slot.ctx != ctx) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_adjoint_scratch) != cudaSuccess || !p) {
            slot = ScratchSlot{};
            return CCS_ERR_CUDA;
        }
        slot.addr = static_cast<float*>(p);
        slot.ctx = known ? ctx : 0;
        if (!known) {                      // not cached: looked up again next time
            *out = slot.addr;
            slot = ScratchSlot{};
            return CCS_OK;
        }
    }
    *out = slot.addr;
    return CCS_OK;
}

}  // namespace ccs

extern "C" int ccs_AdjointPointsDeviceNoAlloc_cuda(cc_Subd* subd, const float* gradPoints, float* gradCage,
                                                   void* stream) {
    using namespace ccs;
    if (!subd || !gradPoints || !gradCage) return set_last_error(CCS_ERR_ARG);
    // the subd's device must be current for the look-up and the launches
    ccs_DeviceArrays arrays;
    if (ccs_GetDeviceArrays_cuda(subd, &arrays) != CCS_OK) return set_last_error(CCS_ERR_ARG);
    if (3 * arrays.vertexCount > kScratchFloats) return set_last_error(CCS_ERR_SCRATCH_LIMIT);
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, arrays.vertexPoints) != cudaSuccess) return set_last_error(CCS_ERR_CUDA);
    DeviceGuard guard(attr.device);        // the caller's device is back on every return
    float* work = nullptr;
    int st = scratch_address(&work);
    if (st == CCS_OK)
        st = adjoint_into(subd, gradPoints, gradCage, work, kScratchFloats, static_cast<cudaStream_t>(stream));
    return set_last_error(st);
}
