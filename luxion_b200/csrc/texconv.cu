// texconv.cu -- texel conversion on the device at scene upload. 8/16-bit unorm texels become
// float (c / 255, c / 65535, the conversion of src/texture.cu:17-27) or binary16, and float
// texels become binary16, so the host uploads the texels as they are (8-bit ones are a quarter
// of the float bytes) and does no per-texel work. The division is IEEE round-to-nearest, as
// the host's, so the texels are the same bit for bit.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/luxion.h"
#include "launch.h"

namespace lux {
namespace {

__device__ __forceinline__ float texel_value(const void* src, int fmt, size_t i) {
    switch (fmt) {
        case LUX_TEX_RGBA8: return __fdiv_rn(float(static_cast<const uint8_t*>(src)[i]), 255.0f);
        case LUX_TEX_RGBA16: return __fdiv_rn(float(static_cast<const uint16_t*>(src)[i]), 65535.0f);
        default: return static_cast<const float*>(src)[i];
    }
}

__global__ void k_texels_to_float(const void* __restrict__ src, int fmt, float* __restrict__ dst, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] = texel_value(src, fmt, i);
}

__global__ void k_texels_to_half(const void* __restrict__ src, int fmt, __half* __restrict__ dst, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] = __float2half_rn(texel_value(src, fmt, i));
}

}  // namespace

cudaError_t launch_convert_texels(const void* src, int fmt, int to_half, void* dst, size_t n, cudaStream_t st) {
    const int grid = int(std::min<size_t>((n + 255) / 256, size_t(148) * 16));
    if (to_half) k_texels_to_half<<<grid, 256, 0, st>>>(src, fmt, static_cast<__half*>(dst), n);
    else k_texels_to_float<<<grid, 256, 0, st>>>(src, fmt, static_cast<float*>(dst), n);
    return cudaGetLastError();
}

}  // namespace lux
