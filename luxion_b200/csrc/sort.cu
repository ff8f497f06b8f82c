// sort.cu -- Morton-keyed ray sorting of a bounce's queue (RAY_SORTING, include/config.h:4).
//
// Keys follow intersectionPrecompute (src/kernels/intersection_precompute.cu:6-33) and
// rayMortonCode / morton3D (src/morton_codes.cu:13-24, include/morton_codes.h:12-38): the
// ray in the first instance's object space, the reference slab test against the Morton box
// (src/mesh/bounding_box.cu:7-40), 0xFFFFFFFF on a miss, else the 30-bit code of the midpoint
// of o and o+d normalised by the box diagonal. Every float operation is rounded on its own,
// so keys are bit-exact with the CPU oracle.
// The reference sorts with thrust::sort_by_key (src/pathtrace.cu:182); here a stable LSD
// radix sort (4 passes of 8 bits) whose length is read from the device counter, so the
// whole bounce stays free of host round trips.

#include "device_scene.h"
#include "device_math.cuh"
#include "launch.h"

#include <algorithm>

namespace lux {
namespace {

constexpr int kSortThreads = 256;
constexpr int kItems = 4;
constexpr int kTile = kSortThreads * kItems;

LUX_DI uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

LUX_DI uint32_t morton3d(float x, float y, float z) {
    x = fminf(fmaxf(__fmul_rn(x, 1024.0f), 0.0f), 1023.0f);
    y = fminf(fmaxf(__fmul_rn(y, 1024.0f), 0.0f), 1023.0f);
    z = fminf(fmaxf(__fmul_rn(z, 1024.0f), 0.0f), 1023.0f);
    return (expand_bits(uint32_t(x)) << 2) | (expand_bits(uint32_t(y)) << 1) | expand_bits(uint32_t(z));
}

LUX_DI uint32_t morton_key(const DevScene& S, f3 o, f3 d) {
    const DevInstance& I = S.insts[0];
    f3 ro = xform(I.Minv, o, 1.0f);
    f3 rd = xform(I.Minv, d, 0.0f);
    f3 inv = mk(__frcp_rn(rd.x), __frcp_rn(rd.y), __frcp_rn(rd.z));
    int sx = inv.x < 0.0f, sy = inv.y < 0.0f, sz = inv.z < 0.0f;
    const float bx[2] = {S.morton_bmin[0], S.morton_bmax[0]};
    const float by[2] = {S.morton_bmin[1], S.morton_bmax[1]};
    const float bz[2] = {S.morton_bmin[2], S.morton_bmax[2]};
    float tmin = __fmul_rn(__fsub_rn(bx[sx], ro.x), inv.x);
    float tmax = __fmul_rn(__fsub_rn(bx[1 - sx], ro.x), inv.x);
    float tymin = __fmul_rn(__fsub_rn(by[sy], ro.y), inv.y);
    float tymax = __fmul_rn(__fsub_rn(by[1 - sy], ro.y), inv.y);
    if (tmin > tymax || tymin > tmax) return 0xFFFFFFFFu;
    tmin = gmax(tmin, tymin);
    tmax = gmin(tmax, tymax);
    float tzmin = __fmul_rn(__fsub_rn(bz[sz], ro.z), inv.z);
    float tzmax = __fmul_rn(__fsub_rn(bz[1 - sz], ro.z), inv.z);
    if (tmin > tzmax || tzmin > tmax) return 0xFFFFFFFFu;
    tmin = gmax(tmin, tzmin);
    if (tmax < 0.0f) return 0xFFFFFFFFu;
    if (!(tmin < tmax)) return 0xFFFFFFFFu;
    f3 ext3 = mk(__fsub_rn(bx[1], bx[0]), __fsub_rn(by[1], by[0]), __fsub_rn(bz[1], bz[0]));
    float ext = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(ext3.x, ext3.x), __fmul_rn(ext3.y, ext3.y)), __fmul_rn(ext3.z, ext3.z)));
    float two = __fmul_rn(2.0f, ext);
    f3 far = mk(__fadd_rn(ro.x, __fmul_rn(rd.x, 1.0f)), __fadd_rn(ro.y, __fmul_rn(rd.y, 1.0f)), __fadd_rn(ro.z, __fmul_rn(rd.z, 1.0f)));
    float p0x = __fdiv_rn(__fadd_rn(ro.x, ext), two), p0y = __fdiv_rn(__fadd_rn(ro.y, ext), two), p0z = __fdiv_rn(__fadd_rn(ro.z, ext), two);
    float p1x = __fdiv_rn(__fadd_rn(far.x, ext), two), p1y = __fdiv_rn(__fadd_rn(far.y, ext), two), p1z = __fdiv_rn(__fadd_rn(far.z, ext), two);
    return morton3d(__fmul_rn(0.5f, __fadd_rn(p0x, p1x)), __fmul_rn(0.5f, __fadd_rn(p0y, p1y)), __fmul_rn(0.5f, __fadd_rn(p0z, p1z)));
}

__global__ void k_keys(DevScene S, DevWave W, int bounce) {
    const int n = *(volatile int*)&W.ctr->count[bounce];
    const int* q = W.queue[bounce & 1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int pid = q[i];
        float4 a = W.s0[pid], b = W.s1[pid];
        W.keys[i] = morton_key(S, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z));
    }
}

__global__ void k_keys_ext(DevScene S, const float* rays, uint32_t* keys, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = rays + size_t(i) * 8;
        keys[i] = morton_key(S, mk(r[0], r[1], r[2]), mk(r[4], r[5], r[6]));
    }
}

// histogram of one 8-bit digit per tile: hist[digit * max_tiles + tile]
__global__ void __launch_bounds__(kSortThreads) k_hist(const uint32_t* keys, const int* nptr, int shift, int* hist,
                                                       int max_tiles) {
    __shared__ int h[256];
    const int n = *(volatile const int*)nptr;
    const int tiles = (n + kTile - 1) / kTile;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        h[threadIdx.x] = 0;
        __syncthreads();
        int base = tile * kTile;
        for (int k = 0; k < kItems; ++k) {
            int i = base + k * kSortThreads + threadIdx.x;
            if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xffu], 1);
        }
        __syncthreads();
        hist[threadIdx.x * max_tiles + tile] = h[threadIdx.x];
        __syncthreads();
    }
}

// exclusive scan over hist in digit-major order (one block)
__global__ void __launch_bounds__(1024) k_scan(int* hist, const int* nptr, int max_tiles) {
    __shared__ int part[1024];
    const int n = *(volatile const int*)nptr;
    const int tiles = (n + kTile - 1) / kTile;
    if (tiles == 0) return;
    const long total = long(tiles) * 256;
    const long per = (total + 1023) / 1024;
    auto at = [&](long j) -> int& { return hist[(j / tiles) * max_tiles + (j % tiles)]; };
    long b = long(threadIdx.x) * per, e = min(total, b + per);
    int s = 0;
    for (long j = b; j < e; ++j) s += at(j);
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (long j = b; j < e; ++j) {
        int v = at(j);
        at(j) = run;
        run += v;
    }
}

// stable scatter: items of a tile keep their order within each digit
__global__ void __launch_bounds__(kSortThreads) k_scatter(const uint32_t* keys, const int* vals, uint32_t* okeys,
                                                          int* ovals, const int* nptr, int shift, const int* hist,
                                                          int max_tiles) {
    __shared__ int base[256];
    __shared__ int cnt[256];
    const int n = *(volatile const int*)nptr;
    const int tiles = (n + kTile - 1) / kTile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        base[threadIdx.x] = hist[threadIdx.x * max_tiles + tile];
        cnt[threadIdx.x] = 0;
        __syncthreads();
        int t0 = tile * kTile;
        // chunks of 32 consecutive items, in order, one warp per chunk
        for (int c = 0; c < kTile / 32; ++c) {
            if ((c % (kSortThreads / 32)) == warp) {
                int i = t0 + c * 32 + lane;
                bool ok = i < n;
                uint32_t key = ok ? keys[i] : 0xffffffffu;
                uint32_t dg = (key >> shift) & 0xffu;
                unsigned peers = __match_any_sync(0xffffffffu, ok ? int(dg) : -1);
                int rank = __popc(peers & lt);
                int leader = __ffs(peers) - 1;
                int b = 0;
                if (ok && lane == leader) b = cnt[dg];
                b = __shfl_sync(0xffffffffu, b, leader);
                if (ok) {
                    int pos = base[dg] + b + rank;
                    okeys[pos] = key;
                    ovals[pos] = vals[i];
                }
                __syncwarp();
                if (ok && lane == leader) cnt[dg] = b + __popc(peers);
            }
            __syncthreads();
        }
        __syncthreads();
    }
}

}  // namespace

size_t morton_sort_temp_bytes(int max_paths) {
    int tiles = (max_paths + kTile - 1) / kTile;
    return size_t(tiles) * 256 * sizeof(int) + 256;
}

cudaError_t launch_morton_sort(const DevScene& S, DevWave& W, int bounce, void* temp, size_t temp_bytes,
                               cudaStream_t st) {
    (void)temp_bytes;
    int max_tiles = (W.max_paths + kTile - 1) / kTile;
    int* hist = static_cast<int*>(temp);
    const int* nptr = &W.ctr->count[bounce];
    k_keys<<<1184, 256, 0, st>>>(S, W, bounce);
    uint32_t* ka = W.keys;
    uint32_t* kb = W.keys_alt;
    int* va = W.queue[bounce & 1];
    int* vb = W.queue_alt;
    int grid = std::max(1, std::min(max_tiles, 148 * 8));
    for (int pass = 0; pass < 4; ++pass) {
        int shift = pass * 8;
        k_hist<<<grid, kSortThreads, 0, st>>>(ka, nptr, shift, hist, max_tiles);
        k_scan<<<1, 1024, 0, st>>>(hist, nptr, max_tiles);
        k_scatter<<<grid, kSortThreads, 0, st>>>(ka, va, kb, vb, nptr, shift, hist, max_tiles);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    // four passes: the sorted queue is back in queue[bounce & 1]
    return cudaGetLastError();
}

cudaError_t launch_morton_ext(const DevScene& S, const float* rays, uint32_t* keys, int n, cudaStream_t st) {
    int grid = std::max(1, std::min((n + 255) / 256, 1184));
    k_keys_ext<<<grid, 256, 0, st>>>(S, rays, keys, n);
    return cudaGetLastError();
}

}  // namespace lux
