/* Force-included before every reference translation unit compiled for the host.
 * It supplies what nvcc would: float overloads of the libm names the device code calls
 * unqualified, __frcp_rn (IEEE reciprocal, = 1.0f/x), the tex2D<float4> fetch (defined by
 * the driver), host thread indices, and an atomicAdd for the survivor counter. */
#pragma once
#include <cmath>
#include <algorithm>
#include <cuda_runtime.h>
using std::isnan; using std::isfinite; using std::max; using std::min; using std::abs;
using std::cos; using std::sin; using std::sqrt; using std::pow;
inline float __frcp_rn(float x) { return 1.0f / x; }
template <class T> T tex2D(cudaTextureObject_t, float, float);
template <> float4 tex2D<float4>(cudaTextureObject_t, float, float);
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
inline int atomicAdd(int* p, int v) { int o = *p; *p += v; return o; }
