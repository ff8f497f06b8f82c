// bvh_gpu.h -- device build of the compressed 8-wide BVH and of the scene geometry around it.
//
// The reference builds its binary BVH on the host (fill_bvh, src/mesh/bvh_build.cu:15-318)
// and, in its active build, hands the triangles to OptiX, which builds on the device
// (src/myoptix/optix_accel.cpp:40-106). Here every BLAS and the TLAS are built by kernels:
// a binned-SAH binary tree (32 bins per axis, cost SA(L)*nL + SA(R)*nR), level by level for
// nodes of more than 32 primitives and one warp per subtree below that, then collapsed into
// 8-wide nodes with quantised child boxes, level by level. The arithmetic is the host
// builder's (bvh_build.cpp) operation for operation, so both produce the same nodes bit for bit.
#pragma once

#include "bvh8.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace lux {

// Result of one build over several independent trees (meshes, or the instances of scenes).
struct DeviceBvh8 {
    BVH8Node* nodes = nullptr;      // device, num_nodes; tree t's nodes are contiguous, in tree order
    uint32_t* leaf_prim = nullptr;  // device, one per primitive: leaf record -> primitive index
    uint32_t num_nodes = 0;
    std::vector<uint32_t> root;     // per tree: node index of its root (node_base added)
    std::vector<uint32_t> count;    // per tree: nodes
    std::vector<int> depth;         // per tree: 8-wide levels (root = 1)
    cudaStream_t stream = nullptr;  // the build's stream: the arrays are freed on it
    DeviceBvh8() = default;
    DeviceBvh8(const DeviceBvh8&) = delete;
    DeviceBvh8& operator=(const DeviceBvh8&) = delete;
    ~DeviceBvh8() { release(); }
    void release();
};

// Stream-ordered scratch from the library's per-device memory pool (freed scratch stays
// reserved for the next build, up to a few GB).
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st);
void scratch_free(void* p, cudaStream_t st);

// Build over n = tree_begin.back() primitive boxes (d_boxes: device, n * 6 floats, min xyz then
// max xyz, padded by the caller). Tree t owns primitives [tree_begin[t], tree_begin[t+1]); it
// must own at least one. Child indices are offset by node_base (the index the first node will
// have in the caller's node array). A node's tri_base is its first leaf record relative to its
// tree's first primitive, or absolute when global_tri_base; the records of tree t occupy
// [tree_begin[t], tree_begin[t+1]) of leaf_prim either way. Returns a LUX_* status.
int build_bvh8_device(const float* d_boxes, const std::vector<int>& tree_begin, uint32_t node_base,
                      bool global_tri_base, cudaStream_t st, DeviceBvh8& out);

// Padded triangle boxes of n triangles in global numbering: triangle p of mesh m = prim_mesh[p]
// has vertices pos[3 * (vert_off[m] + idx[3 p + c])] (idx holds mesh-local vertex indices).
cudaError_t launch_tri_boxes(const float* pos, const uint32_t* idx, const int* prim_mesh, const uint32_t* vert_off,
                             int n, float* boxes, cudaStream_t st);
// prim_mesh[p] = m for p in [tri_off[m], tri_off[m+1]), num_meshes meshes.
cudaError_t launch_fill_mesh_ids(const uint32_t* tri_off, int num_meshes, int* prim_mesh, cudaStream_t st);
// Triangle records in leaf order: record r holds v0 with the mesh-local triangle index in w,
// then e1 = v1 - v0 and e2 = v2 - v0, each rounded once (the values the Moller-Trumbore test
// of src/intersections/mesh_isect.cu:79-82 computes).
cudaError_t launch_tri_records(const uint32_t* leaf_prim, int n, const int* prim_mesh, const uint32_t* tri_off,
                               const uint32_t* vert_off, const float* pos, const uint32_t* idx, float4* prims,
                               cudaStream_t st);
// World boxes of instances. Instance i places mesh inst_mesh[i] by the 3x4 columns M[12 i ..];
// exact: the box of its transformed vertices, else of its transformed mesh-box corners
// (mesh_box: 6 floats per mesh). Evaluated in double, padded, rounded outward to float.
cudaError_t launch_inst_boxes(const float* M, const int* inst_mesh, int num_insts, const float* pos,
                              const uint32_t* vert_off, const float* mesh_box, int exact, float* boxes,
                              cudaStream_t st);
// Single-level layout: padded world boxes of instanced triangles (flat primitive f is triangle
// f - inst_tri_off[i] of instance i = flat_inst[f]; ibox: the instances' padded world boxes),
// and the triangle records in leaf order (object-space v0 / e1 / e2 of the triangle, its
// mesh-local index in v0.w, its instance in e1.w).
cudaError_t launch_flat_boxes(const float* M, const int* inst_mesh, const uint32_t* inst_tri_off, const int* flat_inst,
                              int n, const float* ibox, const float* pos, const uint32_t* idx, const uint32_t* tri_off,
                              const uint32_t* vert_off, float* boxes, cudaStream_t st);
cudaError_t launch_flat_records(const uint32_t* leaf_prim, int n, const int* flat_inst, const uint32_t* inst_tri_off,
                                const int* inst_mesh, const uint32_t* tri_off, const uint32_t* vert_off, const float* pos,
                                const uint32_t* idx, float4* prims, cudaStream_t st);
// Float box of each mesh's vertices (6 floats per mesh).
cudaError_t launch_mesh_boxes(const float* pos, const uint32_t* vert_off, int num_meshes, float* boxes,
                              cudaStream_t st);

}  // namespace lux
