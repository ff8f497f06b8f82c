// bvh8.h -- compressed 8-wide BVH node shared by the host builder and the device traversal.
//
// The reference builds a binary binned-SAH tree with one triangle per leaf and 36-byte AoS
// nodes (src/mesh/bvh_build.cu:15-318, include/mesh/bvh.h:10-28) and, in its active build,
// hands the geometry to OptiX. B200 has no RT cores, so the tree here is the binned-SAH
// binary tree collapsed into 8-wide nodes whose child boxes are quantised to 8 bits per
// plane relative to the node's own box (the compressed wide BVH of Ylitie, Karras and Laine,
// "Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017).
//
// Node: 80 bytes = 5 x 16 B.
//   p[3]       f32   quantisation origin (node box minimum)
//   e[3]       u8    per-axis scale exponent, scale = 2^(e-127)
//   imask      u8    bit s set: slot s holds an internal child
//   child_base u32   index of the first internal child; internal children are stored
//                    contiguously in slot order
//   tri_base   u32   first primitive record of the leaf slots; each leaf slot holds one
//                    primitive, stored in slot order (record = tri_base + rank of the slot
//                    among the leaf slots)
//   meta[8]    u8    meta[0]: bit s set: slot s is a leaf; meta[1..7] zero. A slot in neither
//                    imask nor meta[0] is empty
//   q{lo,hi}{x,y,z}[8] u8  child boxes: lo = p + q*scale (rounded outward at build time)
// Child slots are assigned by the octant of the child centroid around the node centre, so a
// ray visits slots in the order (slot ^ ray_octant) to go near-to-far.
#pragma once
#include <cstdint>

namespace lux {

struct alignas(16) BVH8Node {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(BVH8Node) == 80, "BVH8Node must be 80 bytes");

// one primitive per leaf slot: measured on the 1M-triangle 1080p workload, leaf slots of up to
// 2 or 3 triangles cost more in per-lane triangle tests than they save in node visits
// (traversal 97.5 / 107.6 ms against 83.6 ms per 16-spp step)
constexpr int kMaxLeafPrims = 1;
// Entries of a ray's traversal stack (shared-memory part plus local-memory part, trace.cu). A
// scene build rejects a BVH whose depth could need more.
constexpr int kTraversalStack = 64;

}  // namespace lux

#ifndef __CUDACC__
#include <vector>
namespace lux {
struct BVH8Build {
    std::vector<BVH8Node> nodes;       // root at index 0
    std::vector<uint32_t> prim_order;  // leaf primitive records in node order -> input prim id
    int depth = 0;                     // BVH8 levels (root = 1)
    double sah_cost = 0.0;
};
// boxes: n*6 floats (min xyz, max xyz). The builder pads nothing; callers pad boxes.
void build_bvh8(const float* boxes, int n, BVH8Build& out);
}  // namespace lux
#endif
