// trace_static.cu -- the fixed device scratch behind lux_trace_rays_static.
//
// lux_trace_rays stages a batch of caller rays through three per-call cudaMalloc temporaries
// (rays, hits, the work cursor of the persistent traversal). lux_trace_rays_static stages them
// through this one array instead, compiled into the library, so the call allocates nothing.
// Each device holds its own copy of the array; its address is looked up with
// cudaGetSymbolAddress on every call, with that device current, so a device reset (which
// reloads the module at another address) leaves no stale pointer behind.
#include <cuda_runtime.h>

#include <cstdint>

#include "luxion.h"
#include "launch.h"

namespace lux {
namespace {

constexpr size_t kHeaderBytes = 256;  // work cursor (int) at offset 0, rest unused
constexpr size_t kRayBytes = size_t(LUX_TRACE_STATIC_MAX_RAYS) * 8 * sizeof(float);
constexpr size_t kHitBytes = size_t(LUX_TRACE_STATIC_MAX_RAYS) * 5 * sizeof(uint32_t);
static_assert(kRayBytes % 256 == 0, "hit region starts 256-byte aligned");

static __device__ __align__(256) unsigned char g_trace_scratch[kHeaderBytes + kRayBytes + kHitBytes];

}  // namespace

size_t trace_static_scratch_bytes() { return kHeaderBytes + kRayBytes + kHitBytes; }

cudaError_t trace_static_scratch(int device, TraceScratch& out) {
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    if (cur != device) return cudaErrorInvalidDevice;
    void* base = nullptr;
    e = cudaGetSymbolAddress(&base, g_trace_scratch);
    if (e != cudaSuccess) return e;
    unsigned char* b = static_cast<unsigned char*>(base);
    out.cursor = reinterpret_cast<int*>(b);
    out.rays = reinterpret_cast<float*>(b + kHeaderBytes);
    out.hits = reinterpret_cast<uint32_t*>(b + kHeaderBytes + kRayBytes);
    return cudaSuccess;
}

}  // namespace lux
