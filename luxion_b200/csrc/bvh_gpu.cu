// bvh_gpu.cu -- device build of the compressed 8-wide BVH (bvh_gpu.h).
//
// Binary stage (binned SAH, one primitive per leaf), over all trees at once:
//   * nodes of more than kSmall primitives are split level by level: their ranges are cut into
//     chunks of kChunk primitives, one block per chunk; a pass reduces each node's box and
//     centroid bounds, a pass bins the centroids (32 bins per live axis, shared-memory bins
//     merged into the node's bins with atomic min/max on order-preserving integer keys), one
//     thread per node sweeps the bins in double, and a stable two-pass scatter partitions the
//     node's range;
//   * a node of 2..kSmall primitives is handed to one warp, which builds its whole subtree with
//     one primitive per lane, shuffles for the reductions and the sweep, and a ballot for the
//     stable partition.
// Collapse stage, level by level over the 8-wide levels of all trees at once: one thread per
// 8-wide node opens the child of largest area until 8 slots are filled, assigns slots by child
// centroid octant and quantises the child boxes; exclusive scans give every node's children
// and leaf records their places, breadth first within its tree, trees one after another.
// Every floating-point step is the host builder's (bvh_build.cpp), rounded the same way, and
// every tie is broken the same way, so the nodes are identical to the host build's.

#include "bvh_gpu.h"
#include "host_common.h"

#include <cfloat>
#include <cmath>
#include <map>
#include <mutex>

namespace lux {

// Scratch of the device builds comes from one memory pool per device, owned by the library:
// allocations and frees are stream-ordered (no device-wide synchronisation, as cudaFree has),
// and up to kPoolKeep bytes of freed scratch stay reserved for the next build.
namespace {
constexpr uint64_t kPoolKeep = uint64_t(4) << 30;
std::mutex g_pool_mu;
std::map<int, cudaMemPool_t> g_pools;
}  // namespace

cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        auto it = g_pools.find(dev);
        if (it == g_pools.end()) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
            uint64_t keep = kPoolKeep;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            g_pools[dev] = pool;
        } else {
            pool = it->second;
        }
    }
    cudaError_t r = cudaMallocFromPoolAsync(p, bytes, pool, st);
    if (r == cudaSuccess) note_device_alloc();
    return r;
}

void scratch_free(void* p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
}

namespace {

constexpr int kBins = 32;
constexpr int kSmall = 32;      // nodes of at most this many primitives: one warp per subtree
constexpr int kChunk = 2048;    // primitives per block in the large-node passes
constexpr int kBlock = 256;
constexpr int kPerThread = kChunk / kBlock;
constexpr unsigned FULL = 0xffffffffu;

struct BinNode {
    float lo[3], hi[3];
    int left, right;  // children (-1 for a leaf)
    int begin, count;
};

// Order-preserving map of floats to unsigned keys, for atomic min / max.
__device__ __forceinline__ unsigned fkey(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fval(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ __forceinline__ float cen(float lo, float hi) { return __fmul_rn(0.5f, __fadd_rn(lo, hi)); }

// bin of centroid coordinate c: int((double(c) - lo) * k1), clamped to the bins
__device__ __forceinline__ int bin_of(float c, float lo, double k1) {
    const int b = __double2int_rz(__dmul_rn(__dsub_rn(double(c), double(lo)), k1));
    return min(kBins - 1, max(0, b));
}

// surface area of a float box in double: 2 (dx dy + dy dz + dz dx), extents clamped at 0
__device__ __forceinline__ double area(const float* lo, const float* hi) {
    double d[3];
    for (int a = 0; a < 3; ++a) {
        const double x = __dsub_rn(double(hi[a]), double(lo[a]));
        d[a] = 0.0 < x ? x : 0.0;
    }
    return __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[1]), __dmul_rn(d[1], d[2])), __dmul_rn(d[2], d[0])));
}

// SAH cost area(L) nL + area(R) nR
__device__ __forceinline__ double sah(double al, int nl, double ar, int nr) {
    return __dadd_rn(__dmul_rn(al, double(nl)), __dmul_rn(ar, double(nr)));
}

__device__ __forceinline__ int ceil_log2(double x) {
    int k = 0;
    const double m = frexp(x, &k);
    return m == 0.5 ? k - 1 : k;
}

// ---------------------------------------------------------------------------------------------
// binary stage: set-up
// ---------------------------------------------------------------------------------------------

// Roots: node t is tree t's root; identity order; lists of large and small roots; single-
// primitive trees are leaves at once.
__global__ void k_roots(const float* boxes, const int* tree_begin, int num_trees, BinNode* bn, int* ord0, int* ord_fin,
                        int* large, int* n_large, int* small, int* n_small) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < num_trees; t += gridDim.x * blockDim.x) {
        const int b = tree_begin[t], n = tree_begin[t + 1] - b;
        BinNode& r = bn[t];
        r.begin = b;
        r.count = n;
        r.left = r.right = -1;
        if (n == 1) {
            for (int a = 0; a < 3; ++a) {
                r.lo[a] = boxes[size_t(b) * 6 + a];
                r.hi[a] = boxes[size_t(b) * 6 + 3 + a];
            }
            ord_fin[b] = b;
        } else if (n <= kSmall) {
            for (int i = 0; i < n; ++i) ord_fin[b + i] = b + i;
            small[atomicAdd(n_small, 1)] = t;
        } else {
            large[atomicAdd(n_large, 1)] = t;
        }
    }
}

__global__ void k_iota(int* ord, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) ord[i] = i;
}

// ---------------------------------------------------------------------------------------------
// binary stage: one level of large nodes
// ---------------------------------------------------------------------------------------------

// Per-level-slot state of a large node.
struct Slot {
    unsigned red[12];     // keys: box lo[3], box hi[3], centroid lo[3], centroid hi[3]
    double k1[3];         // bins per unit of centroid extent, 0 for a dead axis
    float clo[3];         // centroid bounds minimum
    int live;             // bit a: axis a has a centroid extent
    int axis, split;      // chosen split: axis and last bin on the left; axis -1: halve by position
    int nl;               // primitives going left
    int chunk0, nchunk;   // the node's chunks in the level's chunk table
};

// Chunk table of the level: chunk c covers [chunk_start[c], +kChunk) of slot chunk_slot[c]'s
// range. One block: per-slot chunk counts, a block-wide exclusive scan, then the entries.
__global__ void __launch_bounds__(1024) k_chunks(const int* level, const int* n_level_ptr, const BinNode* bn,
                                                 Slot* slots, int* chunk_slot, int* chunk_start, int* n_chunks) {
    __shared__ int part[1024];
    const int n_level = *n_level_ptr;
    const int per = (n_level + 1023) / 1024;
    const int s0 = min(n_level, int(threadIdx.x) * per), s1 = min(n_level, s0 + per);
    int sum = 0;
    for (int s = s0; s < s1; ++s) sum += (bn[level[s]].count + kChunk - 1) / kChunk;
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = threadIdx.x >= unsigned(off) ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int c = part[threadIdx.x] - sum;
    for (int s = s0; s < s1; ++s) {
        const BinNode& nd = bn[level[s]];
        const int k = (nd.count + kChunk - 1) / kChunk;
        slots[s].chunk0 = c;
        slots[s].nchunk = k;
        for (int r = 0; r < 12; ++r) slots[s].red[r] = (r < 3 || (r >= 6 && r < 9)) ? 0xffffffffu : 0u;
        for (int j = 0; j < k; ++j) {
            chunk_slot[c + j] = s;
            chunk_start[c + j] = nd.begin + j * kChunk;
        }
        c += k;
    }
    if (threadIdx.x == 1023) *n_chunks = part[1023];
}

__device__ __forceinline__ void load_prim(const float* boxes, int p, float* lo, float* hi) {
    const float* b = boxes + size_t(p) * 6;
    lo[0] = b[0], lo[1] = b[1], lo[2] = b[2];
    hi[0] = b[3], hi[1] = b[4], hi[2] = b[5];
}

// Box and centroid bounds of each large node, merged over its chunks.
__global__ void __launch_bounds__(kBlock) k_reduce(const float* boxes, const int* ord, const int* level, const BinNode* bn,
                                                   Slot* slots, const int* chunk_slot, const int* chunk_start,
                                                   const int* n_chunks) {
    __shared__ unsigned sh[12];
    const int nc = *n_chunks;
    for (int c = blockIdx.x; c < nc; c += gridDim.x) {
        const int s = chunk_slot[c];
        const BinNode& nd = bn[level[s]];
        const int p0 = chunk_start[c], p1 = min(nd.begin + nd.count, p0 + kChunk);
        unsigned r[12];
        for (int k = 0; k < 12; ++k) r[k] = (k < 3 || (k >= 6 && k < 9)) ? 0xffffffffu : 0u;
        for (int i = p0 + threadIdx.x; i < p1; i += kBlock) {
            float lo[3], hi[3];
            load_prim(boxes, ord[i], lo, hi);
            for (int a = 0; a < 3; ++a) {
                const float c3 = cen(lo[a], hi[a]);
                r[a] = min(r[a], fkey(lo[a]));
                r[3 + a] = max(r[3 + a], fkey(hi[a]));
                r[6 + a] = min(r[6 + a], fkey(c3));
                r[9 + a] = max(r[9 + a], fkey(c3));
            }
        }
        for (int k = 0; k < 12; ++k) {
            for (int off = 16; off > 0; off >>= 1) {
                const unsigned o = __shfl_xor_sync(FULL, r[k], off);
                r[k] = (k < 3 || (k >= 6 && k < 9)) ? min(r[k], o) : max(r[k], o);
            }
        }
        if (threadIdx.x < 12) sh[threadIdx.x] = (threadIdx.x < 3 || (threadIdx.x >= 6 && threadIdx.x < 9)) ? 0xffffffffu : 0u;
        __syncthreads();
        if ((threadIdx.x & 31) == 0)
            for (int k = 0; k < 12; ++k) {
                if (k < 3 || (k >= 6 && k < 9)) atomicMin(&sh[k], r[k]);
                else atomicMax(&sh[k], r[k]);
            }
        __syncthreads();
        if (threadIdx.x < 12) {
            const int k = threadIdx.x;
            if (k < 3 || (k >= 6 && k < 9)) atomicMin(&slots[s].red[k], sh[k]);
            else atomicMax(&slots[s].red[k], sh[k]);
        }
        __syncthreads();
    }
}

// Node boxes from the reductions; live axes and bin scales.
__global__ void k_bin_setup(const int* level, const int* n_level_ptr, BinNode* bn, Slot* slots) {
    const int n_level = *n_level_ptr;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_level; s += gridDim.x * blockDim.x) {
        Slot& S = slots[s];
        BinNode& nd = bn[level[s]];
        S.live = 0;
        for (int a = 0; a < 3; ++a) {
            nd.lo[a] = fval(S.red[a]);
            nd.hi[a] = fval(S.red[3 + a]);
            const float clo = fval(S.red[6 + a]), chi = fval(S.red[9 + a]);
            const double ext = __dsub_rn(double(chi), double(clo));
            S.clo[a] = clo;
            if (ext > 0.0) {
                S.live |= 1 << a;
                S.k1[a] = __ddiv_rn(double(kBins), ext);
            } else {
                S.k1[a] = 0.0;
            }
        }
    }
}

// Bins of each large node: counts and boxes per live axis, merged over its chunks.
__global__ void __launch_bounds__(kBlock) k_bin(const float* boxes, const int* ord, const int* level, const BinNode* bn,
                                                const Slot* slots, const int* chunk_slot, const int* chunk_start,
                                                const int* n_chunks, unsigned* bin_cnt, unsigned* bin_lo,
                                                unsigned* bin_hi) {
    __shared__ unsigned cnt[3 * kBins];
    __shared__ unsigned blo[3 * kBins * 3], bhi[3 * kBins * 3];
    const int nc = *n_chunks;
    for (int c = blockIdx.x; c < nc; c += gridDim.x) {
        const int s = chunk_slot[c];
        const Slot& S = slots[s];
        const BinNode& nd = bn[level[s]];
        const int p0 = chunk_start[c], p1 = min(nd.begin + nd.count, p0 + kChunk);
        for (int b = threadIdx.x; b < 3 * kBins; b += kBlock) {
            cnt[b] = 0;
            for (int d = 0; d < 3; ++d) {
                blo[b * 3 + d] = 0xffffffffu;
                bhi[b * 3 + d] = 0u;
            }
        }
        __syncthreads();
        for (int i = p0 + threadIdx.x; i < p1; i += kBlock) {
            float lo[3], hi[3];
            load_prim(boxes, ord[i], lo, hi);
            for (int a = 0; a < 3; ++a) {
                if (!((S.live >> a) & 1)) continue;
                const int b = a * kBins + bin_of(cen(lo[a], hi[a]), S.clo[a], S.k1[a]);
                atomicAdd(&cnt[b], 1u);
                for (int d = 0; d < 3; ++d) {
                    atomicMin(&blo[b * 3 + d], fkey(lo[d]));
                    atomicMax(&bhi[b * 3 + d], fkey(hi[d]));
                }
            }
        }
        __syncthreads();
        for (int b = threadIdx.x; b < 3 * kBins; b += kBlock) {
            if (cnt[b] == 0) continue;
            const size_t g = size_t(s) * 3 * kBins + b;
            atomicAdd(&bin_cnt[g], cnt[b]);
            for (int d = 0; d < 3; ++d) {
                atomicMin(&bin_lo[g * 3 + d], blo[b * 3 + d]);
                atomicMax(&bin_hi[g * 3 + d], bhi[b * 3 + d]);
            }
        }
        __syncthreads();
    }
}

// The host builder's sweep over the non-empty bins of each live axis: the first split of
// lowest cost in (axis, bin) order; no live axis (or a one-sided split) halves the range.
// One warp per node, lane b = bin b: the box and count left of a split after bin b are a
// prefix union over lanes 0..b, those right of it a suffix union over lanes b+1..31 (empty
// bins contribute nothing), so every candidate's cost is the host's value exactly.
constexpr int kSplitWarps = 4;
__global__ void __launch_bounds__(32 * kSplitWarps) k_split(const int* level, const int* n_level_ptr, const BinNode* bn,
                                                             Slot* slots, const unsigned* bin_cnt,
                                                             const unsigned* bin_lo, const unsigned* bin_hi) {
    const int n_level = *n_level_ptr;
    const int lane = threadIdx.x & 31;
    for (int s = blockIdx.x * kSplitWarps + (threadIdx.x >> 5); s < n_level; s += gridDim.x * kSplitWarps) {
        Slot& S = slots[s];
        const BinNode& nd = bn[level[s]];
        double best = DBL_MAX;
        int bax = 3, bsp = kBins, bnl = 0;
        for (int a = 0; a < 3; ++a) {
            if (!((S.live >> a) & 1)) continue;
            const size_t g = size_t(s) * 3 * kBins + size_t(a) * kBins + lane;
            const int n = int(bin_cnt[g]);
            float lo[3], hi[3];
            for (int d = 0; d < 3; ++d) {
                lo[d] = n ? fval(bin_lo[g * 3 + d]) : FLT_MAX;
                hi[d] = n ? fval(bin_hi[g * 3 + d]) : -FLT_MAX;
            }
            // inclusive prefix (left side) and inclusive suffix unions over the lanes
            float pl[3], ph[3], ql[3], qh[3];
            int pc = n, qc = n;
            for (int d = 0; d < 3; ++d) {
                pl[d] = ql[d] = lo[d];
                ph[d] = qh[d] = hi[d];
            }
            for (int off = 1; off < 32; off <<= 1) {
                const int uc = __shfl_up_sync(FULL, pc, off), dc = __shfl_down_sync(FULL, qc, off);
                float ul[3], uh[3], dl[3], dh[3];
                for (int d = 0; d < 3; ++d) {
                    ul[d] = __shfl_up_sync(FULL, pl[d], off);
                    uh[d] = __shfl_up_sync(FULL, ph[d], off);
                    dl[d] = __shfl_down_sync(FULL, ql[d], off);
                    dh[d] = __shfl_down_sync(FULL, qh[d], off);
                }
                if (lane >= off) {
                    pc += uc;
                    for (int d = 0; d < 3; ++d) {
                        pl[d] = fminf(pl[d], ul[d]);
                        ph[d] = fmaxf(ph[d], uh[d]);
                    }
                }
                if (lane + off < 32) {
                    qc += dc;
                    for (int d = 0; d < 3; ++d) {
                        ql[d] = fminf(ql[d], dl[d]);
                        qh[d] = fmaxf(qh[d], dh[d]);
                    }
                }
            }
            // right side of a split after bin b: the suffix from b + 1
            int rc = __shfl_down_sync(FULL, qc, 1);
            float rl[3], rh[3];
            for (int d = 0; d < 3; ++d) {
                rl[d] = __shfl_down_sync(FULL, ql[d], 1);
                rh[d] = __shfl_down_sync(FULL, qh[d], 1);
            }
            if (lane == 31) rc = 0;
            if (n > 0 && rc > 0) {
                const double c = sah(area(pl, ph), pc, area(rl, rh), rc);
                if (c < best) {  // axes ascend, so an earlier axis keeps a tie
                    best = c;
                    bax = a;
                    bsp = lane;
                    bnl = pc;
                }
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double ob = __shfl_xor_sync(FULL, best, off);
            const int oa = __shfl_xor_sync(FULL, bax, off);
            const int os = __shfl_xor_sync(FULL, bsp, off);
            const int on = __shfl_xor_sync(FULL, bnl, off);
            if (ob < best || (ob == best && (oa < bax || (oa == bax && os < bsp)))) {
                best = ob;
                bax = oa;
                bsp = os;
                bnl = on;
            }
        }
        if (lane == 0) {
            int axis = bax < 3 ? bax : -1;
            if (axis >= 0 && (bnl <= 0 || bnl >= nd.count)) axis = -1;
            S.axis = axis;
            S.split = axis >= 0 ? bsp : -1;
            S.nl = axis >= 0 ? bnl : nd.count / 2;
        }
    }
}

__device__ __forceinline__ bool goes_left(const Slot& S, const float* boxes, int p, int rel) {
    if (S.axis < 0) return rel < S.nl;
    const float* b = boxes + size_t(p) * 6;
    const int a = S.axis;
    return bin_of(cen(b[a], b[3 + a]), S.clo[a], S.k1[a]) <= S.split;
}

__global__ void __launch_bounds__(kBlock) k_count_left(const float* boxes, const int* ord, const int* level,
                                                       const BinNode* bn, const Slot* slots, const int* chunk_slot,
                                                       const int* chunk_start, const int* n_chunks, int* chunk_left) {
    __shared__ int sh[kBlock / 32];
    const int nc = *n_chunks;
    for (int c = blockIdx.x; c < nc; c += gridDim.x) {
        const int s = chunk_slot[c];
        const Slot& S = slots[s];
        const BinNode& nd = bn[level[s]];
        const int p0 = chunk_start[c], p1 = min(nd.begin + nd.count, p0 + kChunk);
        int k = 0;
        for (int i = p0 + threadIdx.x; i < p1; i += kBlock) k += goes_left(S, boxes, ord[i], i - nd.begin) ? 1 : 0;
        for (int off = 16; off > 0; off >>= 1) k += __shfl_xor_sync(FULL, k, off);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = k;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < kBlock / 32; ++w) t += sh[w];
            chunk_left[c] = t;
        }
        __syncthreads();
    }
}

// Exclusive prefix of the left counts over each node's chunks.
__global__ void k_chunk_base(const int* n_level_ptr, const Slot* slots, const int* chunk_left, int* chunk_lbase) {
    const int n_level = *n_level_ptr;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_level; s += gridDim.x * blockDim.x) {
        int run = 0;
        for (int j = 0; j < slots[s].nchunk; ++j) {
            chunk_lbase[slots[s].chunk0 + j] = run;
            run += chunk_left[slots[s].chunk0 + j];
        }
    }
}

// Empty bins of the level's nodes: count 0, minimum keys all ones, maximum keys zero.
__global__ void k_bin_clear(const int* n_level_ptr, unsigned* bin_cnt, unsigned* bin_lo, unsigned* bin_hi) {
    const size_t n = size_t(*n_level_ptr) * 3 * kBins;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        bin_cnt[i] = 0u;
        for (int d = 0; d < 3; ++d) {
            bin_lo[i * 3 + d] = 0xffffffffu;
            bin_hi[i * 3 + d] = 0u;
        }
    }
}

// After a level: the next binary ids start past its children, and its list count is cleared
// for the level after next (the two lists alternate).
__global__ void k_level_advance(int* n_level_cur, int* next_id) {
    *next_id += 2 * *n_level_cur;
    *n_level_cur = 0;
}

// Stable partition: each chunk's primitives, in order, to the left or right part of the range.
__global__ void __launch_bounds__(kBlock) k_scatter(const float* boxes, const int* ord, int* ord_next, const int* level,
                                                    const BinNode* bn, const Slot* slots, const int* chunk_slot,
                                                    const int* chunk_start, const int* n_chunks,
                                                    const int* chunk_lbase) {
    __shared__ int sh[kBlock / 32];
    const int nc = *n_chunks;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = blockIdx.x; c < nc; c += gridDim.x) {
        const int s = chunk_slot[c];
        const Slot& S = slots[s];
        const BinNode& nd = bn[level[s]];
        const int p0 = chunk_start[c], p1 = min(nd.begin + nd.count, p0 + kChunk);
        // thread t owns positions p0 + t*kPerThread .. + kPerThread - 1 (in order)
        int prim[kPerThread];
        bool left[kPerThread];
        int mine = 0;
        for (int k = 0; k < kPerThread; ++k) {
            const int i = p0 + int(threadIdx.x) * kPerThread + k;
            prim[k] = i < p1 ? ord[i] : -1;
            left[k] = i < p1 && goes_left(S, boxes, prim[k], i - nd.begin);
            mine += left[k] ? 1 : 0;
        }
        int incl = mine;
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, off);
            if (lane >= off) incl += v;
        }
        if (lane == 31) sh[warp] = incl;
        __syncthreads();
        int wbase = 0;
        for (int w = 0; w < warp; ++w) wbase += sh[w];
        int lrank = chunk_lbase[c] + wbase + incl - mine;   // lefts before this thread's first
        int pos_in_chunk = int(threadIdx.x) * kPerThread;
        const int chunk_rel = p0 - nd.begin;
        for (int k = 0; k < kPerThread; ++k) {
            const int i = p0 + pos_in_chunk + k;
            if (i >= p1) break;
            if (left[k]) {
                ord_next[nd.begin + lrank] = prim[k];
                ++lrank;
            } else {
                const int rrank = (chunk_rel + pos_in_chunk + k) - lrank;  // rights before it in the node
                ord_next[nd.begin + S.nl + rrank] = prim[k];
            }
        }
        __syncthreads();
    }
}

// Children of the level's nodes: ids next_id + 2 s and + 1; leaves take their primitive's box
// at once, small children go to the warp list (their range copied to the final order), large
// children to the next level.
// Child ids continue from *next_id (k_level_advance moves it on); ids past bn_cap set *err
// and the level stops there.
__global__ void k_children(const float* boxes, const int* ord_next, int* ord_fin, const int* level,
                           const int* n_level_ptr, BinNode* bn, const Slot* slots, const int* next_id_ptr,
                           int bn_cap, int* err, int* large_next, int* n_large_next, int* small, int* n_small) {
    const int n_level = *n_level_ptr, next_id = *next_id_ptr;
    if (n_level > 0 && next_id + 2 * n_level > bn_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *err = 1;
        return;
    }
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n_level; s += gridDim.x * blockDim.x) {
        BinNode& nd = bn[level[s]];
        const int nl = slots[s].nl;
        const int ids[2] = {next_id + 2 * s, next_id + 2 * s + 1};
        const int beg[2] = {nd.begin, nd.begin + nl};
        const int cnt[2] = {nl, nd.count - nl};
        nd.left = ids[0];
        nd.right = ids[1];
        for (int k = 0; k < 2; ++k) {
            BinNode& ch = bn[ids[k]];
            ch.begin = beg[k];
            ch.count = cnt[k];
            ch.left = ch.right = -1;
            if (cnt[k] == 1) {
                const int p = ord_next[beg[k]];
                load_prim(boxes, p, ch.lo, ch.hi);
                ord_fin[beg[k]] = p;
            } else if (cnt[k] <= kSmall) {
                for (int i = 0; i < cnt[k]; ++i) ord_fin[beg[k] + i] = ord_next[beg[k] + i];
                small[atomicAdd(n_small, 1)] = ids[k];
            } else {
                large_next[atomicAdd(n_large_next, 1)] = ids[k];
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// binary stage: subtrees of at most kSmall primitives, one warp each
// ---------------------------------------------------------------------------------------------

constexpr int kSmallWarps = 4;

__device__ __forceinline__ float wmin(float v) {
    for (int off = 16; off > 0; off >>= 1) v = fminf(v, __shfl_xor_sync(FULL, v, off));
    return v;
}
__device__ __forceinline__ float wmax(float v) {
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL, v, off));
    return v;
}

__global__ void __launch_bounds__(32 * kSmallWarps) k_small(const float* boxes, const int* small, const int* n_small_ptr,
                                                            BinNode* bn, int* ord_fin, int* bn_next) {
    __shared__ int perm[kSmallWarps][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int n_small = *n_small_ptr;
    const unsigned lt = (1u << lane) - 1u;
    for (int w = blockIdx.x * kSmallWarps + wib; w < n_small; w += gridDim.x * kSmallWarps) {
        const int root = small[w];
        const int begin0 = bn[root].begin, cnt0 = min(bn[root].count, kSmall);   // 2 .. kSmall
        int pid = -1;
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX}, c[3] = {0.f, 0.f, 0.f};
        if (lane < cnt0) {
            pid = ord_fin[begin0 + lane];
            load_prim(boxes, pid, lo, hi);
            for (int a = 0; a < 3; ++a) c[a] = cen(lo[a], hi[a]);
        }
        int next = 0;
        if (lane == 0) next = atomicAdd(bn_next, 2 * cnt0 - 2);
        next = __shfl_sync(FULL, next, 0);
        // stack entry k lives in lane k's registers
        int st_node = 0, st_lb = 0, st_n = 0;
        int sp = 0;
        if (lane == 0) {
            st_node = root;
            st_lb = 0;
            st_n = cnt0;
        }
        sp = 1;
        while (sp > 0) {
            --sp;
            const int node = __shfl_sync(FULL, st_node, sp);
            const int lb = __shfl_sync(FULL, st_lb, sp);
            const int n = __shfl_sync(FULL, st_n, sp);
            const bool in = lane >= lb && lane < lb + n;
            const unsigned inmask = __ballot_sync(FULL, in);
            // box and centroid bounds over the node's lanes
            float nlo[3], nhi[3], clo[3], chi[3];
            for (int a = 0; a < 3; ++a) {
                nlo[a] = wmin(in ? lo[a] : FLT_MAX);
                nhi[a] = wmax(in ? hi[a] : -FLT_MAX);
                clo[a] = wmin(in ? c[a] : FLT_MAX);
                chi[a] = wmax(in ? c[a] : -FLT_MAX);
            }
            if (lane == 0) {
                BinNode& nd = bn[node];
                for (int a = 0; a < 3; ++a) {
                    nd.lo[a] = nlo[a];
                    nd.hi[a] = nhi[a];
                }
            }
            int newpos = lane;  // position after the partition, for lanes of the node
            int mid;
            if (n == 2) {
                // the first axis with a centroid extent decides: the smaller centroid goes left
                bool swap = false;
                for (int a = 0; a < 3; ++a) {
                    if (!(__dsub_rn(double(chi[a]), double(clo[a])) > 0.0)) continue;
                    const float c0 = __shfl_sync(FULL, c[a], lb), c1 = __shfl_sync(FULL, c[a], lb + 1);
                    swap = c1 < c0;
                    break;
                }
                if (swap && in) newpos = lane == lb ? lb + 1 : lb;
                mid = lb + 1;
            } else {
                double k1[3];
                int live = 0;
                for (int a = 0; a < 3; ++a) {
                    const double ext = __dsub_rn(double(chi[a]), double(clo[a]));
                    k1[a] = ext > 0.0 ? __ddiv_rn(double(kBins), ext) : 0.0;
                    if (ext > 0.0) live |= 1 << a;
                }
                int bin[3] = {0, 0, 0};
                for (int a = 0; a < 3; ++a)
                    if (in && ((live >> a) & 1)) bin[a] = bin_of(c[a], clo[a], k1[a]);
                // each lane evaluates the split after its own bin on every live axis
                double best = DBL_MAX;
                int bax = 3, bsp = kBins, bnl = 0;
                bool any = false;
                for (int a = 0; a < 3; ++a) {
                    if (!((live >> a) & 1)) continue;
                    float l_lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, l_hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                    float r_lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, r_hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
                    int nl = 0, nr = 0;
                    for (int m = lb; m < lb + n; ++m) {
                        const int bm = __shfl_sync(FULL, bin[a], m);
                        float mlo[3], mhi[3];
                        for (int d = 0; d < 3; ++d) {
                            mlo[d] = __shfl_sync(FULL, lo[d], m);
                            mhi[d] = __shfl_sync(FULL, hi[d], m);
                        }
                        if (bm <= bin[a]) {
                            for (int d = 0; d < 3; ++d) {
                                l_lo[d] = fminf(l_lo[d], mlo[d]);
                                l_hi[d] = fmaxf(l_hi[d], mhi[d]);
                            }
                            ++nl;
                        } else {
                            for (int d = 0; d < 3; ++d) {
                                r_lo[d] = fminf(r_lo[d], mlo[d]);
                                r_hi[d] = fmaxf(r_hi[d], mhi[d]);
                            }
                            ++nr;
                        }
                    }
                    if (in && nr > 0) {
                        const double cst = sah(area(l_lo, l_hi), nl, area(r_lo, r_hi), nr);
                        if (!any || cst < best) {  // axes ascend, so the first wins ties
                            best = cst;
                            bax = a;
                            bsp = bin[a];
                            bnl = nl;
                            any = true;
                        }
                    }
                }
                // warp arg-min over (cost, axis, bin)
                for (int off = 16; off > 0; off >>= 1) {
                    const double ob = __shfl_xor_sync(FULL, best, off);
                    const int oa = __shfl_xor_sync(FULL, bax, off);
                    const int os = __shfl_xor_sync(FULL, bsp, off);
                    const int on = __shfl_xor_sync(FULL, bnl, off);
                    const bool take = ob < best || (ob == best && (oa < bax || (oa == bax && os < bsp)));
                    if (take) {
                        best = ob;
                        bax = oa;
                        bsp = os;
                        bnl = on;
                    }
                }
                if (bax < 3 && bnl > 0 && bnl < n) {
                    const bool l = in && bin[bax] <= bsp;
                    const unsigned lm = __ballot_sync(FULL, l);
                    const int nl = __popc(lm);
                    if (in) newpos = l ? lb + __popc(lm & lt) : lb + nl + __popc(inmask & ~lm & lt);
                    mid = lb + nl;
                } else {
                    mid = lb + n / 2;  // coincident centroids: halve by position
                }
            }
            // apply the permutation (lanes of the node move to newpos)
            if (in) perm[wib][newpos] = lane;
            __syncwarp();
            const int src = in ? perm[wib][lane] : lane;
            __syncwarp();
            pid = __shfl_sync(FULL, pid, src);
            for (int a = 0; a < 3; ++a) {
                lo[a] = __shfl_sync(FULL, lo[a], src);
                hi[a] = __shfl_sync(FULL, hi[a], src);
                c[a] = __shfl_sync(FULL, c[a], src);
            }
            // children
            const int ids[2] = {next, next + 1};
            next += 2;
            const int clb[2] = {lb, mid};
            const int cn[2] = {mid - lb, lb + n - mid};
            if (lane == 0) {
                bn[node].left = ids[0];
                bn[node].right = ids[1];
            }
            for (int k = 0; k < 2; ++k) {
                if (lane == 0) {
                    BinNode& ch = bn[ids[k]];
                    ch.begin = begin0 + clb[k];
                    ch.count = cn[k];
                    ch.left = ch.right = -1;
                }
                if (cn[k] == 1) {
                    if (lane == clb[k]) {
                        BinNode& ch = bn[ids[k]];
                        for (int a = 0; a < 3; ++a) {
                            ch.lo[a] = lo[a];
                            ch.hi[a] = hi[a];
                        }
                        ord_fin[begin0 + lane] = pid;
                    }
                } else {
                    if (lane == sp) {
                        st_node = ids[k];
                        st_lb = clb[k];
                        st_n = cn[k];
                    }
                    ++sp;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// collapse stage
// ---------------------------------------------------------------------------------------------

struct Item {
    int bnode;
    int tree;
};

// The items a launch works on: [off, off + count) of the level arrays. With lvl set, both come
// from the device level table (lvl[2 l], lvl[2 l + 1]), so that levels are launched back to back
// without the host reading their sizes; otherwise off = 0 and count = n.
struct Span {
    const int* lvl;
    int l;
    int n;
    __device__ int off() const { return lvl ? lvl[2 * l] : 0; }
    __device__ int count() const { return lvl ? lvl[2 * l + 1] : n; }
};

// One 8-wide node per item: its children, slots, quantised boxes (child_base and tri_base are
// placed later), the binary ids of its internal children and the primitives of its leaf slots,
// both in slot order.
__global__ void k_collapse(Span sp, const Item* items_all, const BinNode* bn, const int* ord_fin, BVH8Node* tmp_all,
                           int* n_int_all, int* n_leaf_all, int* child_bn_all, int* leaf_prim_all) {
    const int o = sp.off(), n_items = sp.count();
    const Item* items = items_all + o;
    BVH8Node* tmp = tmp_all + o;
    int *n_int = n_int_all + o, *n_leaf = n_leaf_all + o;
    int *child_bn = child_bn_all + size_t(o) * 8, *leaf_prim = leaf_prim_all + size_t(o) * 8;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x) {
        const BinNode& b = bn[items[it].bnode];
        int ch[8];
        int nch = 0;
        if (b.left < 0 || b.count <= kMaxLeafPrims) {
            ch[nch++] = items[it].bnode;
        } else {
            ch[nch++] = b.left;
            ch[nch++] = b.right;
            while (nch < 8) {
                int pick = -1;
                double pa = -1.0;
                for (int k = 0; k < nch; ++k) {
                    const BinNode& c = bn[ch[k]];
                    if (c.left < 0 || c.count <= kMaxLeafPrims) continue;
                    const double a = area(c.lo, c.hi);
                    if (a > pa) {
                        pa = a;
                        pick = k;
                    }
                }
                if (pick < 0) break;
                const int c = ch[pick];
                ch[pick] = bn[c].left;
                ch[nch++] = bn[c].right;
            }
        }
        // slots by centroid octant around the node centre, cheapest (child, slot) pairs first
        float ctr[3];
        for (int a = 0; a < 3; ++a) ctr[a] = cen(b.lo[a], b.hi[a]);
        double cost[8][8];
        for (int k = 0; k < nch; ++k) {
            const BinNode& c = bn[ch[k]];
            double d[3];
            for (int a = 0; a < 3; ++a)
                d[a] = __dsub_rn(__dmul_rn(0.5, __dadd_rn(double(c.lo[a]), double(c.hi[a]))), double(ctr[a]));
            for (int s = 0; s < 8; ++s) {
                double v = 0.0;
                for (int a = 0; a < 3; ++a) v = __dadd_rn(v, ((s >> a) & 1) ? -d[a] : d[a]);
                cost[k][s] = v;
            }
        }
        int slot_of[8];
        bool slot_used[8] = {false, false, false, false, false, false, false, false};
        bool cdone[8] = {false, false, false, false, false, false, false, false};
        for (int round = 0; round < nch; ++round) {
            int bc = -1, bs = -1;
            double bcost = 0.0;
            for (int k = 0; k < nch; ++k) {
                if (cdone[k]) continue;
                for (int s = 0; s < 8; ++s) {
                    if (slot_used[s]) continue;
                    if (bc < 0 || cost[k][s] < bcost) {
                        bcost = cost[k][s];
                        bc = k;
                        bs = s;
                    }
                }
            }
            cdone[bc] = true;
            slot_used[bs] = true;
            slot_of[bc] = bs;
        }
        int at_slot[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
        for (int k = 0; k < nch; ++k) at_slot[slot_of[k]] = ch[k];
        // quantisation (encode_node of the host builder)
        BVH8Node N;
        {
            uint32_t* w = reinterpret_cast<uint32_t*>(&N);
            for (int k = 0; k < 20; ++k) w[k] = 0;
        }
        double mext = 0.0, mabs = 0.0;
        for (int a = 0; a < 3; ++a) {
            mext = fmax(mext, __dsub_rn(double(b.hi[a]), double(b.lo[a])));
            mabs = fmax(mabs, fmax(fabs(double(b.lo[a])), fabs(double(b.hi[a]))));
        }
        const double pad = __dadd_rn(__dadd_rn(__dmul_rn(1e-4, mext), __dmul_rn(1e-7, mabs)), 1e-30);
        double hi_d[3];
        for (int a = 0; a < 3; ++a) {
            const double lo_d = __dsub_rn(double(b.lo[a]), pad);
            hi_d[a] = __dadd_rn(double(b.hi[a]), pad);
            float pf = __double2float_rn(lo_d);
            if (double(pf) > lo_d) pf = nextafterf(pf, -FLT_MAX);
            N.p[a] = pf;
        }
        for (int a = 0; a < 3; ++a) {
            const double ext = __dsub_rn(hi_d[a], double(N.p[a]));
            int e = -126;
            if (ext > 0.0) e = ceil_log2(__ddiv_rn(ext, 255.0));
            e = max(-126, min(127, e));
            while (ldexp(255.0, e) < ext && e < 127) ++e;
            N.e[a] = uint8_t(e + 127);
        }
        uint8_t* qlo[3] = {N.qlox, N.qloy, N.qloz};
        uint8_t* qhi[3] = {N.qhix, N.qhiy, N.qhiz};
        for (int s = 0; s < 8; ++s) {
            for (int a = 0; a < 3; ++a) {
                if (at_slot[s] < 0) {
                    qlo[a][s] = 0xff;
                    qhi[a][s] = 0x00;
                    continue;
                }
                const BinNode& c = bn[at_slot[s]];
                const double scale = ldexp(1.0, int(N.e[a]) - 127);
                const double l = floor(__dsub_rn(__ddiv_rn(__dsub_rn(double(c.lo[a]), double(N.p[a])), scale), 0.01));
                const double h = ceil(__dadd_rn(__ddiv_rn(__dsub_rn(double(c.hi[a]), double(N.p[a])), scale), 0.01));
                qlo[a][s] = uint8_t(fmax(0.0, fmin(255.0, l)));
                qhi[a][s] = uint8_t(fmax(0.0, fmin(255.0, h)));
            }
        }
        int ni = 0, nl = 0;
        for (int s = 0; s < 8; ++s) {
            const int c = at_slot[s];
            if (c < 0) continue;
            const BinNode& cn = bn[c];
            if (cn.left < 0 || cn.count <= kMaxLeafPrims) {
                leaf_prim[size_t(it) * 8 + nl] = ord_fin[cn.begin];  // one primitive per leaf slot
                ++nl;
                N.meta[0] = uint8_t(N.meta[0] | (1u << s));
            } else {
                N.imask = uint8_t(N.imask | (1u << s));
                child_bn[size_t(it) * 8 + ni] = c;
                ++ni;
            }
        }
        tmp[it] = N;
        n_int[it] = ni;
        n_leaf[it] = nl;
    }
}

// next level: item cs[it] + k is internal child k of item it; the next level starts right
// after this one
__global__ void k_emit(Span sp, Item* items_all, const int* n_int_all, const int* cs_all, const int* child_bn_all,
                       long long cap) {
    const int o = sp.off(), n_items = sp.count();
    const Item* items = items_all + o;
    const int *n_int = n_int_all + o, *cs = cs_all + o;
    const int* child_bn = child_bn_all + size_t(o) * 8;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x)
        for (int k = 0; k < n_int[it]; ++k) {
            const long long at = (long long)o + n_items + cs[it] + k;  // past the capacity: k_level_next flags it
            if (at < cap) items_all[at] = Item{child_bn[size_t(it) * 8 + k], items[it].tree};
        }
}

// Level l + 1 of the table: it starts after level l and holds *n_next items (the total of the
// scan of level l's internal-child counts). Past the capacity it is left empty and err is set.
__global__ void k_level_next(int* lvl, int l, const int* n_next, long long cap, int* err) {
    const long long o = (long long)lvl[2 * l] + lvl[2 * l + 1];
    const int n = *n_next;
    lvl[2 * (l + 1)] = int(o);
    if (o + n > cap) {
        lvl[2 * (l + 1) + 1] = 0;
        *err = 1;
    } else {
        lvl[2 * (l + 1) + 1] = n;
    }
}

// exclusive scan of n ints (in -> out), total to *total; three passes over blocks of 1024
constexpr int kScanBlock = 1024;
__global__ void __launch_bounds__(256) k_scan_local(Span sp, const int* in_all, int* out_all, int* block_sums) {
    __shared__ int sh[256];
    const int o = sp.off(), n = sp.count();
    const int* in = in_all + o;
    int* out = out_all + o;
    const int base = blockIdx.x * kScanBlock;
    if (blockIdx.x > 0 && base >= n) return;  // block 0 always writes its (maybe empty) sum
    int v[4], s = 0;
    for (int k = 0; k < 4; ++k) {
        const int i = base + int(threadIdx.x) * 4 + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
        const int t = threadIdx.x >= unsigned(off) ? sh[threadIdx.x - off] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - s;
    for (int k = 0; k < 4; ++k) {
        const int i = base + int(threadIdx.x) * 4 + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (threadIdx.x == 255) block_sums[blockIdx.x] = sh[255];
}
__global__ void __launch_bounds__(1024) k_scan_sums(Span sp, int* block_sums, int* total) {
    __shared__ int sh[1024];
    const int nb = max(1, (sp.count() + kScanBlock - 1) / kScanBlock);
    const int per = (nb + 1023) / 1024;
    const int b0 = min(nb, int(threadIdx.x) * per), b1 = min(nb, b0 + per);
    int s = 0;
    for (int b = b0; b < b1; ++b) s += block_sums[b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int t = threadIdx.x >= unsigned(off) ? sh[threadIdx.x - off] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - s;
    for (int b = b0; b < b1; ++b) {
        const int v = block_sums[b];
        block_sums[b] = run;
        run += v;
    }
    if (threadIdx.x == 1023) *total = sh[1023];
}
__global__ void k_scan_add(Span sp, int* out_all, const int* block_sums) {
    const int n = sp.count();
    int* out = out_all + sp.off();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] += block_sums[i / kScanBlock];
}

// Where each tree's items of a level start and end: first[t] (atomic min) and last[t] (max).
__global__ void k_bounds(const Item* items, int n_items, int* first, int* last) {
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x) {
        const int t = items[it].tree;
        if (it == 0 || items[it - 1].tree != t) first[t] = it;
        if (it == n_items - 1 || items[it + 1].tree != t) last[t] = it;
    }
}

// Per tree: nodes and leaf records per level -> offsets of each level (nodes absolute, leaf
// records relative to the tree), total nodes and depth. One thread per tree after a scan of the
// trees' node totals (single block).
__global__ void __launch_bounds__(1024) k_tree_offsets(int num_trees, int num_levels, const int* first, const int* last,
                                                       const int* const* ls_level, const int* const* nl_level,
                                                       uint32_t node_base, uint32_t* node_off, uint32_t* leaf_off,
                                                       uint32_t* tree_nodes, int* tree_depth, uint32_t* tree_root) {
    __shared__ uint32_t part[1024];
    const int per = (num_trees + 1023) / 1024;
    const int t0 = min(num_trees, int(threadIdx.x) * per), t1 = min(num_trees, t0 + per);
    uint32_t sum = 0;
    for (int t = t0; t < t1; ++t) {
        uint32_t cnt = 0;
        int depth = 0;
        for (int L = 0; L < num_levels; ++L) {
            const int f = first[size_t(L) * num_trees + t];
            if (f < 0 || last[size_t(L) * num_trees + t] < f) continue;
            cnt += uint32_t(last[size_t(L) * num_trees + t] - f + 1);
            depth = L + 1;
        }
        tree_nodes[t] = cnt;
        tree_depth[t] = depth;
        sum += cnt;
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const uint32_t v = threadIdx.x >= unsigned(off) ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = node_base + part[threadIdx.x] - sum;
    for (int t = t0; t < t1; ++t) {
        tree_root[t] = run;
        uint32_t lrun = 0;
        for (int L = 0; L <= num_levels; ++L) {
            node_off[size_t(L) * num_trees + t] = run;
            leaf_off[size_t(L) * num_trees + t] = lrun;
            if (L == num_levels) break;
            const int f = first[size_t(L) * num_trees + t];
            if (f < 0) continue;
            const int l = last[size_t(L) * num_trees + t];
            if (l < f) continue;
            run += uint32_t(l - f + 1);
            lrun += uint32_t(ls_level[L][l] + nl_level[L][l] - ls_level[L][f]);
        }
    }
}

// Final nodes of one level and their leaf records.
__global__ void k_place(const Item* items, int n_items, int L, int num_trees, const BVH8Node* tmp, const int* cs,
                        const int* ls, const int* n_leaf, const int* leaf_prim, const int* first,
                        const uint32_t* node_off, const uint32_t* leaf_off, const int* tree_begin, bool global_tri,
                        uint32_t node_base, uint32_t total_nodes, BVH8Node* nodes, uint32_t* leaf_out) {
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x) {
        const int t = items[it].tree;
        const int f = first[size_t(L) * num_trees + t];
        const uint32_t idx = node_off[size_t(L) * num_trees + t] + uint32_t(it - f);
        BVH8Node N = tmp[it];
        N.child_base = node_off[size_t(L + 1) * num_trees + t] + uint32_t(cs[it] - cs[f]);
        const uint32_t rec = leaf_off[size_t(L) * num_trees + t] + uint32_t(ls[it] - ls[f]);
        N.tri_base = rec + (global_tri ? uint32_t(tree_begin[t]) : 0u);
        if (idx - node_base < total_nodes) nodes[idx - node_base] = N;
        for (int k = 0; k < n_leaf[it]; ++k) {
            const size_t r = size_t(tree_begin[t]) + rec + k;
            if (r < size_t(tree_begin[t + 1])) leaf_out[r] = uint32_t(leaf_prim[size_t(it) * 8 + k]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// scene geometry
// ---------------------------------------------------------------------------------------------

__global__ void k_fill_mesh_ids(const uint32_t* tri_off, int num_meshes, int* prim_mesh) {
    for (int m = blockIdx.x; m < num_meshes; m += gridDim.x)
        for (uint32_t p = tri_off[m] + threadIdx.x; p < tri_off[m + 1]; p += blockDim.x) prim_mesh[p] = m;
}

__global__ void k_tri_boxes(const float* pos, const uint32_t* idx, const int* prim_mesh, const uint32_t* vert_off, int n,
                            float* boxes) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t vb = vert_off[prim_mesh[p]];
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int c = 0; c < 3; ++c) {
            const float* v = pos + size_t(vb + idx[size_t(p) * 3 + c]) * 3;
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], v[a]);
                hi[a] = fmaxf(hi[a], v[a]);
            }
        }
        float* b = boxes + size_t(p) * 6;
        for (int a = 0; a < 3; ++a) {
            const float pad = __fadd_rn(__fmul_rn(1e-6f, fmaxf(fabsf(lo[a]), fabsf(hi[a]))), 1e-9f);
            b[a] = __fsub_rn(lo[a], pad);
            b[3 + a] = __fadd_rn(hi[a], pad);
        }
    }
}

__global__ void k_tri_records(const uint32_t* leaf_prim, int n, const int* prim_mesh, const uint32_t* tri_off,
                              const uint32_t* vert_off, const float* pos, const uint32_t* idx, float4* out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t p = min(leaf_prim[r], uint32_t(n - 1));
        const int m = prim_mesh[p];
        const uint32_t vb = vert_off[m];
        const float* v0 = pos + size_t(vb + idx[size_t(p) * 3 + 0]) * 3;
        const float* v1 = pos + size_t(vb + idx[size_t(p) * 3 + 1]) * 3;
        const float* v2 = pos + size_t(vb + idx[size_t(p) * 3 + 2]) * 3;
        const int local = int(p - tri_off[m]);
        out[size_t(r) * 3 + 0] = make_float4(v0[0], v0[1], v0[2], __int_as_float(local));
        out[size_t(r) * 3 + 1] = make_float4(__fsub_rn(v1[0], v0[0]), __fsub_rn(v1[1], v0[1]), __fsub_rn(v1[2], v0[2]), 0.0f);
        out[size_t(r) * 3 + 2] = make_float4(__fsub_rn(v2[0], v0[0]), __fsub_rn(v2[1], v0[1]), __fsub_rn(v2[2], v0[2]), 0.0f);
    }
}

__global__ void k_mesh_boxes(const float* pos, const uint32_t* vert_off, int num_meshes, float* boxes) {
    __shared__ float sh[6][32];
    for (int m = blockIdx.x; m < num_meshes; m += gridDim.x) {
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t v = vert_off[m] + threadIdx.x; v < vert_off[m + 1]; v += blockDim.x)
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(lo[a], pos[size_t(v) * 3 + a]);
                hi[a] = fmaxf(hi[a], pos[size_t(v) * 3 + a]);
            }
        for (int a = 0; a < 3; ++a) {
            lo[a] = wmin(lo[a]);
            hi[a] = wmax(hi[a]);
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0)
            for (int a = 0; a < 3; ++a) {
                sh[a][w] = lo[a];
                sh[3 + a][w] = hi[a];
            }
        __syncthreads();
        if (threadIdx.x < 6) {
            float r = threadIdx.x < 3 ? FLT_MAX : -FLT_MAX;
            for (int k = 0; k < nw; ++k) r = threadIdx.x < 3 ? fminf(r, sh[threadIdx.x][k]) : fmaxf(r, sh[threadIdx.x][k]);
            boxes[size_t(m) * 6 + threadIdx.x] = r;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ double dmin_w(double v) {
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(FULL, v, off));
    return v;
}
__device__ __forceinline__ double dmax_w(double v) {
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, off));
    return v;
}

__global__ void k_inst_boxes(const float* M, const int* inst_mesh, int num_insts, const float* pos, const uint32_t* vert_off,
                             const float* mesh_box, int exact, float* boxes) {
    __shared__ double sh[6][32];
    for (int i = blockIdx.x; i < num_insts; i += gridDim.x) {
        const float* T = M + size_t(i) * 12;
        const int m = inst_mesh[i];
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        auto grow = [&](double x, double y, double z) {
            for (int a = 0; a < 3; ++a) {
                const double w = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(double(T[0 * 3 + a]), x), __dmul_rn(double(T[1 * 3 + a]), y)),
                                                     __dmul_rn(double(T[2 * 3 + a]), z)),
                                           double(T[3 * 3 + a]));
                lo[a] = fmin(lo[a], w);
                hi[a] = fmax(hi[a], w);
            }
        };
        if (exact) {
            for (uint32_t v = vert_off[m] + threadIdx.x; v < vert_off[m + 1]; v += blockDim.x)
                grow(pos[size_t(v) * 3], pos[size_t(v) * 3 + 1], pos[size_t(v) * 3 + 2]);
        } else if (threadIdx.x < 8) {
            const float* mb = mesh_box + size_t(m) * 6;
            const int c = threadIdx.x;
            grow((c & 1) ? mb[3] : mb[0], (c & 2) ? mb[4] : mb[1], (c & 4) ? mb[5] : mb[2]);
        }
        for (int a = 0; a < 3; ++a) {
            lo[a] = dmin_w(lo[a]);
            hi[a] = dmax_w(hi[a]);
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        if (lane == 0)
            for (int a = 0; a < 3; ++a) {
                sh[a][w] = lo[a];
                sh[3 + a][w] = hi[a];
            }
        __syncthreads();
        if (threadIdx.x == 0) {
            double L[3], H[3];
            for (int a = 0; a < 3; ++a) {
                L[a] = 1e300;
                H[a] = -1e300;
                for (int k = 0; k < nw; ++k) {
                    L[a] = fmin(L[a], sh[a][k]);
                    H[a] = fmax(H[a], sh[3 + a][k]);
                }
            }
            double mext = 0, mabs = 0;
            for (int a = 0; a < 3; ++a) {
                mext = fmax(mext, __dsub_rn(H[a], L[a]));
                mabs = fmax(mabs, fmax(fabs(L[a]), fabs(H[a])));
            }
            const double pad = __dadd_rn(__dadd_rn(__dmul_rn(1e-5, mext), __dmul_rn(1e-6, mabs)), 1e-12);
            for (int a = 0; a < 3; ++a) {
                boxes[size_t(i) * 6 + a] = __double2float_rn(__dsub_rn(L[a], pad));
                boxes[size_t(i) * 6 + 3 + a] = __double2float_rn(__dadd_rn(H[a], pad));
            }
        }
        __syncthreads();
    }
}

// World boxes of instanced triangles for the single-level layout: flat primitive f is
// triangle k = f - inst_tri_off[i] of instance i = flat_inst[f]. The box of the triangle's
// vertices transformed in double is padded by 1e-5 of the instance's world extent plus 1e-5 of
// its largest coordinate (ibox: the instance's padded world box): the object-space triangle
// test sees the ray through the instance's float inverse, whose point error grows with the
// coordinates' magnitude, and the pad covers it for condition numbers up to about 20.
__global__ void k_flat_boxes(const float* M, const int* inst_mesh, const uint32_t* inst_tri_off, const int* flat_inst,
                             int n, const float* ibox, const float* pos, const uint32_t* idx, const uint32_t* tri_off,
                             const uint32_t* vert_off, float* boxes) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
        const int i = flat_inst[f];
        const int m = inst_mesh[i];
        const uint32_t p = tri_off[m] + (uint32_t(f) - inst_tri_off[i]);
        const float* T = M + size_t(i) * 12;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int c = 0; c < 3; ++c) {
            const float* v = pos + size_t(vert_off[m] + idx[size_t(p) * 3 + c]) * 3;
            for (int a = 0; a < 3; ++a) {
                const double w = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(double(T[0 * 3 + a]), double(v[0])),
                                                               __dmul_rn(double(T[1 * 3 + a]), double(v[1]))),
                                                     __dmul_rn(double(T[2 * 3 + a]), double(v[2]))),
                                           double(T[3 * 3 + a]));
                lo[a] = fmin(lo[a], w);
                hi[a] = fmax(hi[a], w);
            }
        }
        const float* ib = ibox + size_t(i) * 6;
        double mext = 0.0, mabs = 0.0;
        for (int a = 0; a < 3; ++a) {
            mext = fmax(mext, __dsub_rn(double(ib[3 + a]), double(ib[a])));
            mabs = fmax(mabs, fmax(fabs(double(ib[a])), fabs(double(ib[3 + a]))));
        }
        const double pad = __dadd_rn(__dmul_rn(1e-5, __dadd_rn(mext, mabs)), 1e-12);
        for (int a = 0; a < 3; ++a) {
            boxes[size_t(f) * 6 + a] = __double2float_rd(__dsub_rn(lo[a], pad));
            boxes[size_t(f) * 6 + 3 + a] = __double2float_ru(__dadd_rn(hi[a], pad));
        }
    }
}

// Single-level triangle records in leaf order: v0 with the mesh-local triangle index in w,
// e1 with the instance index in w, e2 -- object-space values, exactly those of the two-level
// records, so the triangle test is the same.
__global__ void k_flat_records(const uint32_t* leaf_prim, int n, const int* flat_inst, const uint32_t* inst_tri_off,
                               const int* inst_mesh, const uint32_t* tri_off, const uint32_t* vert_off, const float* pos,
                               const uint32_t* idx, float4* out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t f = min(leaf_prim[r], uint32_t(n - 1));
        const int i = flat_inst[f];
        const int m = inst_mesh[i];
        const uint32_t k = f - inst_tri_off[i];
        const uint32_t p = tri_off[m] + k;
        const uint32_t vb = vert_off[m];
        const float* v0 = pos + size_t(vb + idx[size_t(p) * 3 + 0]) * 3;
        const float* v1 = pos + size_t(vb + idx[size_t(p) * 3 + 1]) * 3;
        const float* v2 = pos + size_t(vb + idx[size_t(p) * 3 + 2]) * 3;
        out[size_t(r) * 3 + 0] = make_float4(v0[0], v0[1], v0[2], __int_as_float(int(k)));
        out[size_t(r) * 3 + 1] = make_float4(__fsub_rn(v1[0], v0[0]), __fsub_rn(v1[1], v0[1]), __fsub_rn(v1[2], v0[2]),
                                             __int_as_float(i));
        out[size_t(r) * 3 + 2] = make_float4(__fsub_rn(v2[0], v0[0]), __fsub_rn(v2[1], v0[1]), __fsub_rn(v2[2], v0[2]), 0.0f);
    }
}

// device buffers of one build, freed together
struct Bufs {
    cudaStream_t st;
    std::vector<void*> p;
    explicit Bufs(cudaStream_t s) : st(s) {}
    ~Bufs() {
        for (void* q : p) scratch_free(q, st);
    }
    template <class T>
    T* get(size_t n) {
        void* q = nullptr;
        if (scratch_alloc(&q, std::max<size_t>(n, 1) * sizeof(T), st) != cudaSuccess) return nullptr;
        p.push_back(q);
        return static_cast<T*>(q);
    }
};

int grid_for(int n, int per_block, int cap) { return std::max(1, std::min(cap, (n + per_block - 1) / per_block)); }

// exclusive scan of n device ints (in -> out); the total lands in *total (device)
// Exclusive scan of sp's items of in into out (both indexed from the level start); max_n bounds
// the count for the launch shapes. The block sums need max(1, ceil(max_n / kScanBlock)) ints.
int device_scan(Span sp, int max_n, const int* in, int* out, int* total, int* block_sums, cudaStream_t st) {
    const int nb = std::max(1, (max_n + kScanBlock - 1) / kScanBlock);
    k_scan_local<<<nb, 256, 0, st>>>(sp, in, out, block_sums);
    k_scan_sums<<<1, 1024, 0, st>>>(sp, block_sums, total);
    k_scan_add<<<grid_for(max_n, 256, 4096), 256, 0, st>>>(sp, out, block_sums);
    LUX_CUDA(cudaGetLastError());
    return LUX_OK;
}

}  // namespace

void DeviceBvh8::release() {
    scratch_free(nodes, stream);
    scratch_free(leaf_prim, stream);
    nodes = nullptr;
    leaf_prim = nullptr;
    num_nodes = 0;
}

int build_bvh8_device(const float* d_boxes, const std::vector<int>& tree_begin, uint32_t node_base, bool global_tri,
                      cudaStream_t st, DeviceBvh8& out) {
    out.release();
    const int G = int(tree_begin.size()) - 1;
    if (G <= 0) return fail(LUX_ERR_INVALID, "BVH build without trees");
    for (int t = 0; t < G; ++t)
        if (tree_begin[t + 1] <= tree_begin[t]) return fail(LUX_ERR_INVALID, "BVH build: a tree without primitives");
    const int N = tree_begin[G];
    Bufs B(st);
    int* d_tb = B.get<int>(G + 1);
    int* ord[2] = {B.get<int>(N), B.get<int>(N)};
    int* ord_fin = B.get<int>(N);
    const size_t bn_cap = size_t(2) * N;
    BinNode* bn = B.get<BinNode>(bn_cap);
    const int large_cap = N / (kSmall + 1) + 1;
    int* large[2] = {B.get<int>(large_cap), B.get<int>(large_cap)};
    int* small = B.get<int>(N / 2 + 1);
    int* ctr = B.get<int>(8);  // 0,1: large list sizes; 2: small list size; 3: next binary id; 4: chunks
    Slot* slots = B.get<Slot>(large_cap);
    unsigned* bin_cnt = B.get<unsigned>(size_t(large_cap) * 3 * kBins);
    unsigned* bin_lo = B.get<unsigned>(size_t(large_cap) * 3 * kBins * 3);
    unsigned* bin_hi = B.get<unsigned>(size_t(large_cap) * 3 * kBins * 3);
    const int chunk_cap = large_cap + N / kChunk + 1;
    int* chunk_slot = B.get<int>(chunk_cap);
    int* chunk_start = B.get<int>(chunk_cap);
    int* chunk_left = B.get<int>(chunk_cap);
    int* chunk_lbase = B.get<int>(chunk_cap);
    int* h_ctr = nullptr;
    if (!d_tb || !ord[0] || !ord[1] || !ord_fin || !bn || !large[0] || !large[1] || !small || !ctr || !slots ||
        !bin_cnt || !bin_lo || !bin_hi || !chunk_slot || !chunk_start || !chunk_left || !chunk_lbase)
        return fail(LUX_ERR_OOM, "BVH build: device scratch allocation failed");
    h_ctr = static_cast<int*>(pinned_get(8 * sizeof(int)));
    if (!h_ctr) return fail(LUX_ERR_OOM, "BVH build: page-locked host allocation failed");
    struct HostFree {  // back to the pool once no copy into it can still be queued
        int* p;
        cudaStream_t st;
        ~HostFree() {
            cudaStreamSynchronize(st);
            pinned_put(p, 8 * sizeof(int));
        }
    } hf{h_ctr, st};
    LUX_CUDA(cudaMemcpyAsync(d_tb, tree_begin.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    LUX_CUDA(cudaMemsetAsync(ctr, 0, 8 * sizeof(int), st));
    // every index array starts in range, so no read can leave its buffer whatever is computed
    LUX_CUDA(cudaMemsetAsync(ord[1], 0, sizeof(int) * size_t(N), st));
    LUX_CUDA(cudaMemsetAsync(ord_fin, 0, sizeof(int) * size_t(N), st));
    LUX_CUDA(cudaMemsetAsync(bn, 0, sizeof(BinNode) * bn_cap, st));
    k_iota<<<grid_for(N, 256, 4096), 256, 0, st>>>(ord[0], N);
    k_roots<<<grid_for(G, 128, 1024), 128, 0, st>>>(d_boxes, d_tb, G, bn, ord[0], ord_fin, large[0], ctr + 0, small,
                                                   ctr + 2);
    LUX_CUDA(cudaGetLastError());
    LUX_CUDA(cudaMemcpyAsync(h_ctr, ctr, 8 * sizeof(int), cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaStreamSynchronize(st));
    // Binary levels of large nodes, launched in batches without reading their sizes back:
    // every kernel takes the level's node count from ctr[cur] (the two large lists alternate),
    // binary ids continue from ctr[3], and a level past the last has no nodes, so its kernels
    // do nothing. One read-back per batch finds the first empty level; ctr[7] flags a binary
    // node table too small.
    h_ctr[3] = G;
    LUX_CUDA(cudaMemcpyAsync(ctr + 3, h_ctr + 3, sizeof(int), cudaMemcpyHostToDevice, st));
    int max_tree = 1;
    for (int t = 0; t < G; ++t) max_tree = std::max(max_tree, tree_begin[t + 1] - tree_begin[t]);
    const int grid_s = grid_for(large_cap, 128, 4096);
    const int grid_sp = grid_for(large_cap, kSplitWarps, 4096);
    const int grid_clear = grid_for(large_cap * 3 * kBins, 256, 148 * 16);
    const int grid_c = std::min(chunk_cap, 148 * 8);
    int cur = 0, levels = 0;
    int batch = int(std::ceil(std::log2(double(max_tree) / double(kSmall) + 1.0))) + 2;
    while (true) {
        for (int b = 0; b < batch; ++b) {
            if (++levels > 4 * 64 + N) return fail(LUX_ERR_UNSUPPORTED, "BVH build did not converge");
            const int nxt = cur ^ 1;
            k_chunks<<<1, 1024, 0, st>>>(large[cur], ctr + cur, bn, slots, chunk_slot, chunk_start, ctr + 4);
            k_bin_clear<<<grid_clear, 256, 0, st>>>(ctr + cur, bin_cnt, bin_lo, bin_hi);
            k_reduce<<<grid_c, kBlock, 0, st>>>(d_boxes, ord[cur], large[cur], bn, slots, chunk_slot, chunk_start,
                                                ctr + 4);
            k_bin_setup<<<grid_s, 128, 0, st>>>(large[cur], ctr + cur, bn, slots);
            k_bin<<<grid_c, kBlock, 0, st>>>(d_boxes, ord[cur], large[cur], bn, slots, chunk_slot, chunk_start, ctr + 4,
                                              bin_cnt, bin_lo, bin_hi);
            k_split<<<grid_sp, 32 * kSplitWarps, 0, st>>>(large[cur], ctr + cur, bn, slots, bin_cnt, bin_lo, bin_hi);
            k_count_left<<<grid_c, kBlock, 0, st>>>(d_boxes, ord[cur], large[cur], bn, slots, chunk_slot, chunk_start,
                                                     ctr + 4, chunk_left);
            k_chunk_base<<<grid_s, 128, 0, st>>>(ctr + cur, slots, chunk_left, chunk_lbase);
            k_scatter<<<grid_c, kBlock, 0, st>>>(d_boxes, ord[cur], ord[nxt], large[cur], bn, slots, chunk_slot,
                                                  chunk_start, ctr + 4, chunk_lbase);
            k_children<<<grid_s, 128, 0, st>>>(d_boxes, ord[nxt], ord_fin, large[cur], ctr + cur, bn, slots, ctr + 3,
                                               int(bn_cap), ctr + 7, large[nxt], ctr + nxt, small, ctr + 2);
            k_level_advance<<<1, 1, 0, st>>>(ctr + cur, ctr + 3);
            LUX_CUDA(cudaGetLastError());
            cur = nxt;
        }
        LUX_CUDA(cudaMemcpyAsync(h_ctr, ctr, 8 * sizeof(int), cudaMemcpyDeviceToHost, st));
        LUX_CUDA(cudaStreamSynchronize(st));
        if (h_ctr[7]) return fail(LUX_ERR_UNSUPPORTED, "BVH build: binary node capacity");
        if (h_ctr[cur] == 0) break;
        batch = 4;
    }
    // small subtrees: binary ids continue after the large levels' children
    const int n_small = h_ctr[2];
    if (n_small > 0) {
        int* nid = ctr + 3;  // the next binary id, past every large level's children
        k_small<<<grid_for(n_small, kSmallWarps, 148 * 16), 32 * kSmallWarps, 0, st>>>(d_boxes, small, ctr + 2, bn,
                                                                                        ord_fin, nid);
        LUX_CUDA(cudaGetLastError());
    }

    // ---- collapse, level by level ----
    const size_t item_cap = size_t(N) + G;
    Item* items = B.get<Item>(item_cap);
    BVH8Node* tmp = B.get<BVH8Node>(item_cap);
    int* n_int = B.get<int>(item_cap);
    int* n_leaf = B.get<int>(item_cap);
    int* cs = B.get<int>(item_cap);
    int* ls = B.get<int>(item_cap);
    int* child_bn = B.get<int>(item_cap * 8);
    int* leafp = B.get<int>(item_cap * 8);
    int* block_sums = B.get<int>(item_cap / kScanBlock + 2);
    if (!items || !tmp || !n_int || !n_leaf || !cs || !ls || !child_bn || !leafp || !block_sums)
        return fail(LUX_ERR_OOM, "BVH build: device scratch allocation failed");
    {
        std::vector<Item> roots(G);
        for (int t = 0; t < G; ++t) roots[t] = Item{t, t};
        LUX_CUDA(cudaMemcpyAsync(items, roots.data(), sizeof(Item) * G, cudaMemcpyHostToDevice, st));
    }
    // The levels are launched in batches without reading their sizes back: every kernel takes
    // its level's offset and count from the device level table (lvl: offset, count per level;
    // then an error word), and a level past the last is empty, so its kernels do nothing. One
    // read-back of the table per batch finds the first empty level. The first batch covers the
    // levels a tree of the largest size usually has (about one 8-wide level per three binary
    // levels of a binary depth near 1.5 log2 n).
    constexpr int kMaxLevels = 120;
    int* lvl = B.get<int>(2 * kMaxLevels + 4);
    int* h_lvl = static_cast<int*>(pinned_get(sizeof(int) * (2 * kMaxLevels + 4)));
    struct LevelFree {
        int* p;
        cudaStream_t st;
        ~LevelFree() {
            cudaStreamSynchronize(st);
            pinned_put(p, sizeof(int) * (2 * kMaxLevels + 4));
        }
    } lf{h_lvl, st};
    if (!lvl || !h_lvl) return fail(LUX_ERR_OOM, "BVH build: level table allocation failed");
    int* lvl_err = lvl + 2 * kMaxLevels + 2;
    LUX_CUDA(cudaMemsetAsync(lvl, 0, sizeof(int) * (2 * kMaxLevels + 4), st));
    {
        const int first[2] = {0, G};
        LUX_CUDA(cudaMemcpyAsync(lvl, first, sizeof(first), cudaMemcpyHostToDevice, st));
        LUX_CUDA(cudaStreamSynchronize(st));  // `first` lives on this stack frame
    }
    const int max_n = int(item_cap);
    const int grid_items = grid_for(max_n, 128, 148 * 16);
    int launched = 0, L = -1;
    batch = int(std::ceil(0.5 * std::log2(double(max_tree) + 1.0))) + 1;
    while (L < 0) {
        batch = std::min(batch, kMaxLevels - launched);
        if (batch <= 0) return fail(LUX_ERR_UNSUPPORTED, "BVH build: too many 8-wide levels");
        for (int l = launched; l < launched + batch; ++l) {
            const Span sp{lvl, l, 0};
            k_collapse<<<grid_items, 128, 0, st>>>(sp, items, bn, ord_fin, tmp, n_int, n_leaf, child_bn, leafp);
            LUX_CUDA(cudaGetLastError());
            if (int rc = device_scan(sp, max_n, n_leaf, ls, ctr + 5, block_sums, st)) return rc;
            if (int rc = device_scan(sp, max_n, n_int, cs, ctr + 6, block_sums, st)) return rc;
            k_level_next<<<1, 1, 0, st>>>(lvl, l, ctr + 6, (long long)item_cap, lvl_err);
            k_emit<<<grid_items, 128, 0, st>>>(sp, items, n_int, cs, child_bn, (long long)item_cap);
            LUX_CUDA(cudaGetLastError());
        }
        launched += batch;
        LUX_CUDA(cudaMemcpyAsync(h_lvl, lvl, sizeof(int) * (2 * kMaxLevels + 4), cudaMemcpyDeviceToHost, st));
        LUX_CUDA(cudaStreamSynchronize(st));
        if (h_lvl[2 * kMaxLevels + 2]) return fail(LUX_ERR_UNSUPPORTED, "BVH build: 8-wide node capacity");
        for (int l = 1; l <= launched; ++l)
            if (h_lvl[2 * l + 1] == 0) {
                L = l;
                break;
            }
        batch = 3;
    }
    std::vector<size_t> lvl_off(L);
    std::vector<int> lvl_n(L);
    for (int l = 0; l < L; ++l) {
        lvl_off[l] = size_t(h_lvl[2 * l]);
        lvl_n[l] = h_lvl[2 * l + 1];
    }
    const size_t total_items = lvl_off.back() + size_t(lvl_n.back());

    // ---- placement ----
    int* first = B.get<int>(size_t(L) * G);
    int* last = B.get<int>(size_t(L) * G);
    uint32_t* node_off = B.get<uint32_t>(size_t(L + 1) * G);
    uint32_t* leaf_off = B.get<uint32_t>(size_t(L + 1) * G);
    uint32_t* tree_nodes = B.get<uint32_t>(G);
    int* tree_depth = B.get<int>(G);
    uint32_t* tree_root = B.get<uint32_t>(G);
    const int** lsp = B.get<const int*>(L);
    const int** nlp = B.get<const int*>(L);
    if (!first || !last || !node_off || !leaf_off || !tree_nodes || !tree_depth || !tree_root || !lsp || !nlp)
        return fail(LUX_ERR_OOM, "BVH build: device scratch allocation failed");
    LUX_CUDA(cudaMemsetAsync(first, 0xff, sizeof(int) * size_t(L) * G, st));
    LUX_CUDA(cudaMemsetAsync(last, 0xff, sizeof(int) * size_t(L) * G, st));
    std::vector<const int*> h_lsp(L), h_nlp(L);
    for (int l = 0; l < L; ++l) {
        h_lsp[l] = ls + lvl_off[l];
        h_nlp[l] = n_leaf + lvl_off[l];
        k_bounds<<<grid_for(lvl_n[l], 128, 4096), 128, 0, st>>>(items + lvl_off[l], lvl_n[l], first + size_t(l) * G,
                                                               last + size_t(l) * G);
    }
    LUX_CUDA(cudaMemcpyAsync(lsp, h_lsp.data(), sizeof(int*) * L, cudaMemcpyHostToDevice, st));
    LUX_CUDA(cudaMemcpyAsync(nlp, h_nlp.data(), sizeof(int*) * L, cudaMemcpyHostToDevice, st));
    k_tree_offsets<<<1, 1024, 0, st>>>(G, L, first, last, lsp, nlp, node_base, node_off, leaf_off, tree_nodes,
                                       tree_depth, tree_root);
    LUX_CUDA(cudaGetLastError());
    out.stream = st;
    if (scratch_alloc(reinterpret_cast<void**>(&out.nodes), sizeof(BVH8Node) * std::max<size_t>(total_items, 1), st) !=
            cudaSuccess ||
        scratch_alloc(reinterpret_cast<void**>(&out.leaf_prim), sizeof(uint32_t) * size_t(N), st) != cudaSuccess) {
        out.release();
        return fail(LUX_ERR_OOM, "BVH build: node allocation failed");
    }
    LUX_CUDA(cudaMemsetAsync(out.leaf_prim, 0, sizeof(uint32_t) * size_t(N), st));
    for (int l = 0; l < L; ++l)
        k_place<<<grid_for(lvl_n[l], 128, 4096), 128, 0, st>>>(items + lvl_off[l], lvl_n[l], l, G, tmp + lvl_off[l],
                                                              cs + lvl_off[l], ls + lvl_off[l], n_leaf + lvl_off[l],
                                                              leafp + lvl_off[l] * 8, first, node_off, leaf_off, d_tb,
                                                              global_tri, node_base, uint32_t(total_items), out.nodes,
                                                              out.leaf_prim);
    LUX_CUDA(cudaGetLastError());
    out.root.resize(G);
    out.count.resize(G);
    out.depth.resize(G);
    LUX_CUDA(cudaMemcpyAsync(out.root.data(), tree_root, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaMemcpyAsync(out.count.data(), tree_nodes, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaMemcpyAsync(out.depth.data(), tree_depth, sizeof(int) * G, cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaStreamSynchronize(st));
    out.num_nodes = uint32_t(total_items);
    return LUX_OK;
}

cudaError_t launch_fill_mesh_ids(const uint32_t* tri_off, int num_meshes, int* prim_mesh, cudaStream_t st) {
    if (num_meshes <= 0) return cudaSuccess;
    k_fill_mesh_ids<<<std::min(num_meshes, 4096), 256, 0, st>>>(tri_off, num_meshes, prim_mesh);
    return cudaGetLastError();
}

cudaError_t launch_tri_boxes(const float* pos, const uint32_t* idx, const int* prim_mesh, const uint32_t* vert_off, int n,
                             float* boxes, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_tri_boxes<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(pos, idx, prim_mesh, vert_off, n, boxes);
    return cudaGetLastError();
}

cudaError_t launch_tri_records(const uint32_t* leaf_prim, int n, const int* prim_mesh, const uint32_t* tri_off,
                               const uint32_t* vert_off, const float* pos, const uint32_t* idx, float4* prims,
                               cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_tri_records<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(leaf_prim, n, prim_mesh, tri_off, vert_off, pos, idx, prims);
    return cudaGetLastError();
}

cudaError_t launch_flat_boxes(const float* M, const int* inst_mesh, const uint32_t* inst_tri_off, const int* flat_inst,
                              int n, const float* ibox, const float* pos, const uint32_t* idx, const uint32_t* tri_off,
                              const uint32_t* vert_off, float* boxes, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_flat_boxes<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(M, inst_mesh, inst_tri_off, flat_inst, n, ibox, pos, idx,
                                                             tri_off, vert_off, boxes);
    return cudaGetLastError();
}

cudaError_t launch_flat_records(const uint32_t* leaf_prim, int n, const int* flat_inst, const uint32_t* inst_tri_off,
                                const int* inst_mesh, const uint32_t* tri_off, const uint32_t* vert_off, const float* pos,
                                const uint32_t* idx, float4* prims, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_flat_records<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(leaf_prim, n, flat_inst, inst_tri_off, inst_mesh, tri_off,
                                                               vert_off, pos, idx, prims);
    return cudaGetLastError();
}

cudaError_t launch_mesh_boxes(const float* pos, const uint32_t* vert_off, int num_meshes, float* boxes, cudaStream_t st) {
    if (num_meshes <= 0) return cudaSuccess;
    k_mesh_boxes<<<std::min(num_meshes, 4096), 256, 0, st>>>(pos, vert_off, num_meshes, boxes);
    return cudaGetLastError();
}

cudaError_t launch_inst_boxes(const float* M, const int* inst_mesh, int num_insts, const float* pos,
                              const uint32_t* vert_off, const float* mesh_box, int exact, float* boxes,
                              cudaStream_t st) {
    if (num_insts <= 0) return cudaSuccess;
    k_inst_boxes<<<std::min(num_insts, 4096), 256, 0, st>>>(M, inst_mesh, num_insts, pos, vert_off, mesh_box, exact,
                                                            boxes);
    return cudaGetLastError();
}

}  // namespace lux
