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
// once per device, with that device current.
static constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mu;
static float* g_scratch_addr[kMaxDevices] = {};

static int scratch_address(float** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CCS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_adjoint_scratch) != cudaSuccess || !p) return CCS_ERR_CUDA;
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_addr[dev];
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
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != attr.device) cudaSetDevice(attr.device);
    float* work = nullptr;
    int st = scratch_address(&work);
    if (st == CCS_OK)
        st = adjoint_into(subd, gradPoints, gradCage, work, kScratchFloats, static_cast<cudaStream_t>(stream));
    if (prev >= 0 && prev != attr.device) cudaSetDevice(prev);
    return set_last_error(st);
}
