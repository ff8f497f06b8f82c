// geometry.cpp -- device geometry of one or more scenes: vertex data uploaded once, every mesh's
// BLAS and every scene's TLAS built by the device BVH builder (bvh_gpu.cu), triangle records
// and instance records, all concatenated into one set of arrays (DevScene).
//
// The reference uploads each mesh and builds its acceleration structures at load
// (Mesh::make_mesh_device, src/mesh/mesh_device.cu:11-45; the OptiX GAS/IAS builds,
// src/myoptix/optix_accel.cpp:9-110, src/myoptix/optix_ias.cpp:9-63; called from
// src/main.cpp:199-274). Here the only host work is the instance records (matrix inverses) and
// the bookkeeping of offsets; vertex data goes from the caller's arrays straight to its place
// in the concatenated device arrays.

#include "bvh_gpu.h"
#include "host_common.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

namespace lux {

namespace {

bool invert4(const float* m, double* out) {
    double t[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            t[r][c] = m[c * 4 + r];
            t[r][c + 4] = (r == c) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(t[r][c]) > std::fabs(t[p][c])) p = r;
        if (std::fabs(t[p][c]) < 1e-300) return false;
        for (int k = 0; k < 8; ++k) std::swap(t[c][k], t[p][k]);
        double d = t[c][c];
        for (int k = 0; k < 8; ++k) t[c][k] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                double f = t[r][c];
                for (int k = 0; k < 8; ++k) t[r][k] -= f * t[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out[c * 4 + r] = t[r][c + 4];
    return true;
}

// Page-locked staging of the vertex uploads, kept for the process and grown on demand: the
// caller's arrays (pageable or not) are gathered into it by host threads, so the upload is a
// few large DMA copies instead of one small copy per mesh array. One build uses it at a time.
constexpr size_t kStageLimit = size_t(2) << 30;
struct PinnedStage {
    std::mutex mu;
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = bytes + bytes / 4;
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = want;
        return e;
    }
};
PinnedStage g_stage;

// Run fn(lo, hi) over [0, n) split into contiguous ranges, one per host thread.
template <class F>
void parallel_ranges(int n, F fn) {
    unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    nt = std::max(1u, std::min(nt, unsigned(n)));
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(fn, int(int64_t(n) * t / nt), int(int64_t(n) * (t + 1) / nt));
    fn(0, int(int64_t(n) / nt));
    for (auto& t : th) t.join();
}

// Scratch device memory of one geometry build (stream-ordered, from the build pool).
struct Scratch {
    cudaStream_t st;
    std::vector<void*> p;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch() {
        for (void* q : p) scratch_free(q, st);
    }
    template <class T>
    int get(T** out, size_t n) {
        void* q = nullptr;
        cudaError_t e = scratch_alloc(&q, std::max<size_t>(n, 1) * sizeof(T), st);
        if (e != cudaSuccess) return fail(LUX_ERR_OOM, std::string("scratch allocation: ") + cudaGetErrorString(e));
        p.push_back(q);
        *out = static_cast<T*>(q);
        return LUX_OK;
    }
};

}  // namespace

int build_geometry(const lux_scene_desc* const* scenes, int ns, const std::vector<int>& material_base, int layout,
                   const DevAlloc& alloc, cudaStream_t st, DevScene& S, GeometryBuild& G) {
    const auto t0 = std::chrono::steady_clock::now();
    // ---- offsets of the concatenation ----
    std::vector<int> mesh_base(size_t(ns) + 1, 0);
    G.inst_base.assign(size_t(ns) + 1, 0);
    for (int s = 0; s < ns; ++s) {
        mesh_base[s + 1] = mesh_base[s] + scenes[s]->num_meshes;
        G.inst_base[s + 1] = G.inst_base[s] + scenes[s]->num_instances;
    }
    const int NM = mesh_base[ns], NI = G.inst_base[ns];
    std::vector<const lux_mesh_desc*> mesh(NM);
    for (int s = 0; s < ns; ++s)
        for (int m = 0; m < scenes[s]->num_meshes; ++m) mesh[mesh_base[s] + m] = &scenes[s]->meshes[m];
    std::vector<uint32_t> tri_off(size_t(NM) + 1, 0), vert_off(size_t(NM) + 1, 0);
    bool any_n = false, any_uv = false;
    for (int m = 0; m < NM; ++m) {
        tri_off[m + 1] = tri_off[m] + uint32_t(mesh[m]->num_tris);
        vert_off[m + 1] = vert_off[m] + uint32_t(mesh[m]->num_verts);
        if (uint64_t(tri_off[m]) + uint64_t(mesh[m]->num_tris) >= (uint64_t(1) << 31))
            return fail(LUX_ERR_UNSUPPORTED, "more than 2^31 triangles");
        any_n |= mesh[m]->normals != nullptr;
        any_uv |= mesh[m]->uvs != nullptr;
    }
    const size_t T = tri_off[NM], V = vert_off[NM];
    // Layout: the single-level world BVH (no instance transitions during traversal) unless
    // instancing makes its per-instance triangle records large: more than 2x the meshes'
    // triangles and more than 16M of them.
    size_t instanced = 0;
    for (int s = 0; s < ns; ++s)
        for (int i = 0; i < scenes[s]->num_instances; ++i)
            instanced += size_t(mesh[mesh_base[s] + scenes[s]->instances[i].mesh]->num_tris);
    if (instanced >= (size_t(1) << 31)) return fail(LUX_ERR_UNSUPPORTED, "more than 2^31 instanced triangles");
    const bool flat = layout == LUX_BVH_SINGLE_LEVEL ||
                      (layout == LUX_BVH_AUTO && (instanced <= 2 * T || instanced <= (size_t(16) << 20)));
    G.bytes = 0;
    auto own = [&](auto** p, size_t n, size_t elem) -> int {
        G.bytes += n * elem;
        return alloc(reinterpret_cast<void**>(p), n * elem);
    };

    // ---- vertex data: gathered into page-locked staging by host threads, then four DMA
    // copies (one per array); above the staging limit each mesh's arrays are copied directly ----
    float *pos = nullptr, *nrm = nullptr, *uv = nullptr;
    uint32_t* idx = nullptr;
    if (int rc = own(&pos, V * 3, sizeof(float))) return rc;
    if (any_n)
        if (int rc = own(&nrm, V * 3, sizeof(float))) return rc;
    if (any_uv)
        if (int rc = own(&uv, V * 2, sizeof(float))) return rc;
    if (int rc = own(&idx, T * 3, sizeof(uint32_t))) return rc;
    const size_t b_pos = V * 12, b_nrm = nrm ? V * 12 : 0, b_uv = uv ? V * 8 : 0, b_idx = T * 12;
    const size_t total = b_pos + b_nrm + b_uv + b_idx;
    std::unique_lock<std::mutex> stage_lock(g_stage.mu);
    if (total <= kStageLimit && g_stage.reserve(total) == cudaSuccess) {
        char* h = static_cast<char*>(g_stage.p);
        char *h_pos = h, *h_nrm = h + b_pos, *h_uv = h_nrm + b_nrm, *h_idx = h_uv + b_uv;
        parallel_ranges(NM, [&](int m0, int m1) {
            for (int m = m0; m < m1; ++m) {
                const lux_mesh_desc& md = *mesh[m];
                const size_t nv = size_t(md.num_verts), nt = size_t(md.num_tris);
                std::memcpy(h_pos + size_t(vert_off[m]) * 12, md.positions, nv * 12);
                std::memcpy(h_idx + size_t(tri_off[m]) * 12, md.indices, nt * 12);
                if (nrm) {
                    if (md.normals) std::memcpy(h_nrm + size_t(vert_off[m]) * 12, md.normals, nv * 12);
                    else std::memset(h_nrm + size_t(vert_off[m]) * 12, 0, nv * 12);
                }
                if (uv) {
                    if (md.uvs) std::memcpy(h_uv + size_t(vert_off[m]) * 8, md.uvs, nv * 8);
                    else std::memset(h_uv + size_t(vert_off[m]) * 8, 0, nv * 8);
                }
            }
        });
        LUX_CUDA(cudaMemcpyAsync(pos, h_pos, b_pos, cudaMemcpyHostToDevice, st));
        if (nrm) LUX_CUDA(cudaMemcpyAsync(nrm, h_nrm, b_nrm, cudaMemcpyHostToDevice, st));
        if (uv) LUX_CUDA(cudaMemcpyAsync(uv, h_uv, b_uv, cudaMemcpyHostToDevice, st));
        LUX_CUDA(cudaMemcpyAsync(idx, h_idx, b_idx, cudaMemcpyHostToDevice, st));
    } else {
        for (int m = 0; m < NM; ++m) {
            const lux_mesh_desc& md = *mesh[m];
            const size_t nv = size_t(md.num_verts), nt = size_t(md.num_tris);
            LUX_CUDA(cudaMemcpyAsync(pos + size_t(vert_off[m]) * 3, md.positions, nv * 12, cudaMemcpyHostToDevice, st));
            LUX_CUDA(cudaMemcpyAsync(idx + size_t(tri_off[m]) * 3, md.indices, nt * 12, cudaMemcpyHostToDevice, st));
            if (nrm) {
                if (md.normals) LUX_CUDA(cudaMemcpyAsync(nrm + size_t(vert_off[m]) * 3, md.normals, nv * 12, cudaMemcpyHostToDevice, st));
                else LUX_CUDA(cudaMemsetAsync(nrm + size_t(vert_off[m]) * 3, 0, nv * 12, st));
            }
            if (uv) {
                if (md.uvs) LUX_CUDA(cudaMemcpyAsync(uv + size_t(vert_off[m]) * 2, md.uvs, nv * 8, cudaMemcpyHostToDevice, st));
                else LUX_CUDA(cudaMemsetAsync(uv + size_t(vert_off[m]) * 2, 0, nv * 8, st));
            }
        }
    }
    LUX_CUDA(cudaStreamSynchronize(st));
    stage_lock.unlock();
    G.ms_upload = ms_since(t0);
    // ---- BLAS of every mesh (two-level layout) ----
    Scratch X(st);
    uint32_t *d_tri_off = nullptr, *d_vert_off = nullptr;
    float* mesh_box = nullptr;
    if (int rc = X.get(&d_tri_off, size_t(NM) + 1)) return rc;
    if (int rc = X.get(&d_vert_off, size_t(NM) + 1)) return rc;
    if (int rc = X.get(&mesh_box, size_t(NM) * 6)) return rc;
    LUX_CUDA(cudaMemcpyAsync(d_tri_off, tri_off.data(), sizeof(uint32_t) * (NM + 1), cudaMemcpyHostToDevice, st));
    LUX_CUDA(cudaMemcpyAsync(d_vert_off, vert_off.data(), sizeof(uint32_t) * (NM + 1), cudaMemcpyHostToDevice, st));
    DeviceBvh8 blas;
    float4* prims = nullptr;
    if (!flat) {
        int* prim_mesh = nullptr;
        float* boxes = nullptr;
        if (int rc = X.get(&prim_mesh, T)) return rc;
        if (int rc = X.get(&boxes, T * 6)) return rc;
        LUX_CUDA(launch_fill_mesh_ids(d_tri_off, NM, prim_mesh, st));
        LUX_CUDA(launch_tri_boxes(pos, idx, prim_mesh, d_vert_off, int(T), boxes, st));
        std::vector<int> tb(tri_off.begin(), tri_off.end());
        if (int rc = build_bvh8_device(boxes, tb, 0, false, st, blas)) return rc;
        if (int rc = own(&prims, T * 3, sizeof(float4))) return rc;
        LUX_CUDA(launch_tri_records(blas.leaf_prim, int(T), prim_mesh, d_tri_off, d_vert_off, pos, idx, prims, st));
    }
    LUX_CUDA(cudaStreamSynchronize(st));
    G.ms_blas = ms_since(t0) - G.ms_upload;
    // ---- instances ----
    std::vector<DevInstance> insts(NI);
    std::vector<float> M12(size_t(NI) * 12);
    std::vector<int> inst_mesh(NI);
    G.instanced_tris.assign(ns, 0);
    G.max_blas_depth.assign(ns, 0);
    for (int s = 0; s < ns; ++s) {
        const lux_scene_desc& d = *scenes[s];
        for (int i = 0; i < d.num_instances; ++i) {
            const lux_instance_desc& in = d.instances[i];
            const int gm = mesh_base[s] + in.mesh;
            DevInstance& I = insts[G.inst_base[s] + i];
            std::memset(&I, 0, sizeof(I));
            float inv[16], invT[16];
            if (in.has_inverse) {
                std::memcpy(inv, in.inverse, 64);
                std::memcpy(invT, in.inv_transpose, 64);
            } else {
                double id[16];
                if (!invert4(in.transform, id)) return fail(LUX_ERR_INVALID, "singular instance transform");
                for (int k = 0; k < 16; ++k) inv[k] = float(id[k]);
                for (int c = 0; c < 4; ++c)
                    for (int r = 0; r < 4; ++r) invT[c * 4 + r] = float(id[r * 4 + c]);
            }
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 3; ++r) {
                    I.M[c * 3 + r] = in.transform[c * 4 + r];
                    I.Minv[c * 3 + r] = inv[c * 4 + r];
                    I.MinvT[c * 3 + r] = invT[c * 4 + r];
                }
            std::memcpy(&M12[size_t(G.inst_base[s] + i) * 12], I.M, sizeof(I.M));
            inst_mesh[G.inst_base[s] + i] = gm;
            const lux_mesh_desc& md = *mesh[gm];
            I.mesh = in.mesh;
            I.material = in.material + material_base[s];
            I.blas_root = flat ? 0u : blas.root[gm];
            I.prim_base = tri_off[gm];
            I.vert_base = vert_off[gm];
            I.idx_base = tri_off[gm];
            const lux_material_desc& mat = d.materials[in.material];
            I.flags = (md.normals ? kInstHasNormals : 0) | (md.uvs ? kInstHasUVs : 0) |
                      (mat.alpha_mode != LUX_ALPHA_OPAQUE ? kInstAnyHit : 0);
            I.num_tris = md.num_tris;
            I.key = i;
            G.instanced_tris[s] += md.num_tris;
            if (!flat) G.max_blas_depth[s] = std::max(G.max_blas_depth[s], blas.depth[gm]);
        }
    }
    DevInstance* d_insts = nullptr;
    if (int rc = own(&d_insts, size_t(NI), sizeof(DevInstance))) return rc;
    LUX_CUDA(cudaMemcpyAsync(d_insts, insts.data(), sizeof(DevInstance) * NI, cudaMemcpyHostToDevice, st));

    // ---- TLAS of every scene ----
    // World boxes of the instances, in double and padded. Each is the exact box of the mesh's
    // transformed vertices: for rotated meshes it is much tighter than the box of the
    // transformed mesh-box corners (measured on the 1M-triangle scene of 200 rotated
    // instances: traversal per 16-spp step 67.8 against 78.6 ms, BVH8 node visits plus
    // triangle tests per camera ray 16.6 against 20.5). Above 64M vertex transforms in a scene
    // (heavily instanced scenes) its instances take the corner boxes instead.
    float *d_M = nullptr, *ibox = nullptr;
    int* d_inst_mesh = nullptr;
    if (int rc = X.get(&d_M, size_t(NI) * 12)) return rc;
    if (int rc = X.get(&d_inst_mesh, size_t(NI))) return rc;
    if (int rc = X.get(&ibox, size_t(NI) * 6)) return rc;
    LUX_CUDA(cudaMemcpyAsync(d_M, M12.data(), sizeof(float) * M12.size(), cudaMemcpyHostToDevice, st));
    LUX_CUDA(cudaMemcpyAsync(d_inst_mesh, inst_mesh.data(), sizeof(int) * NI, cudaMemcpyHostToDevice, st));
    LUX_CUDA(launch_mesh_boxes(pos, d_vert_off, NM, mesh_box, st));
    for (int s = 0; s < ns; ++s) {
        size_t vertex_work = 0;
        for (int i = G.inst_base[s]; i < G.inst_base[s + 1]; ++i) vertex_work += size_t(mesh[inst_mesh[i]]->num_verts);
        const int exact = vertex_work <= (size_t(64) << 20) ? 1 : 0;
        const int i0 = G.inst_base[s], n = G.inst_base[s + 1] - i0;
        LUX_CUDA(launch_inst_boxes(d_M + size_t(i0) * 12, d_inst_mesh + i0, n, pos, d_vert_off, mesh_box, exact,
                                   ibox + size_t(i0) * 6, st));
    }
    if (flat) {
        // ---- single-level layout: one world-space BVH per scene over its instanced triangles ----
        std::vector<uint32_t> itri(size_t(NI) + 1, 0);
        for (int i = 0; i < NI; ++i) itri[i + 1] = itri[i] + uint32_t(mesh[inst_mesh[i]]->num_tris);
        const size_t NT = itri[NI];
        uint32_t* d_itri = nullptr;
        int* flat_inst = nullptr;
        float* fbox = nullptr;
        if (int rc = X.get(&d_itri, size_t(NI) + 1)) return rc;
        if (int rc = X.get(&flat_inst, NT)) return rc;
        if (int rc = X.get(&fbox, NT * 6)) return rc;
        LUX_CUDA(cudaMemcpyAsync(d_itri, itri.data(), sizeof(uint32_t) * (NI + 1), cudaMemcpyHostToDevice, st));
        LUX_CUDA(launch_fill_mesh_ids(d_itri, NI, flat_inst, st));
        LUX_CUDA(launch_flat_boxes(d_M, d_inst_mesh, d_itri, flat_inst, int(NT), ibox, pos, idx, d_tri_off, d_vert_off,
                                   fbox, st));
        std::vector<int> tb(size_t(ns) + 1);
        for (int s = 0; s <= ns; ++s) tb[s] = int(itri[G.inst_base[s]]);
        DeviceBvh8 world;
        if (int rc = build_bvh8_device(fbox, tb, 0, true, st, world)) return rc;
        // a node visit pushes at most two entries (the node's remaining children and a
        // postponed triangle group), so a traversal holds at most 2 * depth + 1
        for (int s = 0; s < ns; ++s)
            if (2 * world.depth[s] + 1 > kTraversalStack)
                return fail(LUX_ERR_UNSUPPORTED, "acceleration structure deeper than the traversal stack");
        BVH8Node* nodes = nullptr;
        float4* fprims = nullptr;
        if (int rc = own(&nodes, world.num_nodes, sizeof(BVH8Node))) return rc;
        if (int rc = own(&fprims, NT * 3, sizeof(float4))) return rc;
        LUX_CUDA(cudaMemcpyAsync(nodes, world.nodes, sizeof(BVH8Node) * world.num_nodes, cudaMemcpyDeviceToDevice, st));
        LUX_CUDA(launch_flat_records(world.leaf_prim, int(NT), flat_inst, d_itri, d_inst_mesh, d_tri_off, d_vert_off, pos,
                                     idx, fprims, st));
        LUX_CUDA(cudaStreamSynchronize(st));
        G.ms_total = ms_since(t0);
        G.ms_tlas = G.ms_total - G.ms_upload - G.ms_blas;
        S.nodes = reinterpret_cast<const uint4*>(nodes);
        S.prims = fprims;
        S.insts = d_insts;
        S.tlas_prims = nullptr;
        S.tlas_leaf = nullptr;
        S.tlas_root = world.root[0];
        S.num_insts = NI;
        S.single_level = 1;
        S.pos = pos;
        S.nrm = nrm;
        S.uv = uv;
        S.idx = idx;
        G.tlas_root = world.root;
        G.blas_nodes = 0;
        G.tlas_nodes = world.num_nodes;
        G.single_level = true;
        return LUX_OK;
    }
    DeviceBvh8 tlas;
    {
        std::vector<int> tb(G.inst_base.begin(), G.inst_base.end());
        if (int rc = build_bvh8_device(ibox, tb, blas.num_nodes, true, st, tlas)) return rc;
    }
    // two per level of either tree, and three at the instance entry (the world-level group, the
    // rest of the TLAS leaf group and the marker)
    for (int s = 0; s < ns; ++s)
        if (2 * (tlas.depth[s] + G.max_blas_depth[s]) + 3 > kTraversalStack)
            return fail(LUX_ERR_UNSUPPORTED, "acceleration structure deeper than the traversal stack");

    // ---- final arrays: BLAS nodes then TLAS nodes; TLAS leaf records ----
    const size_t nn = size_t(blas.num_nodes) + tlas.num_nodes;
    BVH8Node* nodes = nullptr;
    if (int rc = own(&nodes, nn, sizeof(BVH8Node))) return rc;
    LUX_CUDA(cudaMemcpyAsync(nodes, blas.nodes, sizeof(BVH8Node) * blas.num_nodes, cudaMemcpyDeviceToDevice, st));
    LUX_CUDA(cudaMemcpyAsync(nodes + blas.num_nodes, tlas.nodes, sizeof(BVH8Node) * tlas.num_nodes,
                             cudaMemcpyDeviceToDevice, st));
    uint32_t* tlas_prims = nullptr;
    if (int rc = own(&tlas_prims, size_t(NI), sizeof(uint32_t))) return rc;
    LUX_CUDA(cudaMemcpyAsync(tlas_prims, tlas.leaf_prim, sizeof(uint32_t) * NI, cudaMemcpyDeviceToDevice, st));
    std::vector<uint32_t> h_tp(NI);
    LUX_CUDA(cudaMemcpyAsync(h_tp.data(), tlas.leaf_prim, sizeof(uint32_t) * NI, cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaStreamSynchronize(st));
    std::vector<float4> leaf(size_t(NI) * 4);
    for (int k = 0; k < NI; ++k) {
        if (h_tp[k] >= uint32_t(NI)) return fail(LUX_ERR_UNSUPPORTED, "TLAS leaf order out of range");
        const DevInstance& I = insts[h_tp[k]];
        float4* q = &leaf[size_t(k) * 4];
        q[0] = make_float4(I.Minv[0], I.Minv[1], I.Minv[2], I.Minv[3]);
        q[1] = make_float4(I.Minv[4], I.Minv[5], I.Minv[6], I.Minv[7]);
        q[2] = make_float4(I.Minv[8], I.Minv[9], I.Minv[10], I.Minv[11]);
        const uint32_t e[4] = {I.blas_root, I.prim_base, uint32_t(I.flags), h_tp[k]};
        std::memcpy(&q[3], e, 16);
    }
    float4* tlas_leaf = nullptr;
    if (int rc = own(&tlas_leaf, leaf.size(), sizeof(float4))) return rc;
    LUX_CUDA(cudaMemcpyAsync(tlas_leaf, leaf.data(), sizeof(float4) * leaf.size(), cudaMemcpyHostToDevice, st));
    LUX_CUDA(cudaStreamSynchronize(st));

    G.ms_total = ms_since(t0);
    G.ms_tlas = G.ms_total - G.ms_upload - G.ms_blas;
    S.nodes = reinterpret_cast<const uint4*>(nodes);
    S.prims = prims;
    S.insts = d_insts;
    S.tlas_prims = tlas_prims;
    S.tlas_leaf = tlas_leaf;
    S.tlas_root = tlas.root[0];
    S.num_insts = NI;
    S.single_level = 0;
    S.pos = pos;
    S.nrm = nrm;
    S.uv = uv;
    S.idx = idx;
    G.tlas_root = tlas.root;
    G.blas_nodes = blas.num_nodes;
    G.tlas_nodes = tlas.num_nodes;
    G.single_level = false;
    return LUX_OK;
}

}  // namespace lux

extern "C" int lux_bvh8_build(const float* boxes, const int* tree_begin, int num_trees, int on_device, void* nodes,
                              int capacity, uint32_t* order, uint32_t* roots, int* depth, int* num_nodes) {
    using namespace lux;
    if (!boxes || !tree_begin || num_trees <= 0 || !nodes || capacity < 0 || !order || !roots || !depth || !num_nodes)
        return fail(LUX_ERR_INVALID, "bad arguments");
    for (int t = 0; t < num_trees; ++t)
        if (tree_begin[t + 1] <= tree_begin[t] || tree_begin[0] != 0) return fail(LUX_ERR_INVALID, "empty or unordered tree");
    const int n = tree_begin[num_trees];
    BVH8Node* out = static_cast<BVH8Node*>(nodes);
    *num_nodes = 0;
    if (!on_device) {
        uint32_t base = 0;
        for (int t = 0; t < num_trees; ++t) {
            BVH8Build b;
            build_bvh8(boxes + size_t(tree_begin[t]) * 6, tree_begin[t + 1] - tree_begin[t], b);
            if (base + b.nodes.size() > size_t(capacity)) return fail(LUX_ERR_INVALID, "node capacity too small");
            for (size_t k = 0; k < b.nodes.size(); ++k) {
                out[base + k] = b.nodes[k];
                out[base + k].child_base += base;
            }
            for (size_t k = 0; k < b.prim_order.size(); ++k) order[tree_begin[t] + k] = uint32_t(tree_begin[t]) + b.prim_order[k];
            roots[t] = base;
            depth[t] = b.depth;
            base += uint32_t(b.nodes.size());
        }
        *num_nodes = int(base);
        return LUX_OK;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(LUX_ERR_NO_DEVICE, "no CUDA device");
    cudaStream_t st = nullptr;
    LUX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamFree {
        cudaStream_t s;
        ~StreamFree() { cudaStreamDestroy(s); }
    } sf{st};
    Scratch X(st);
    float* d_boxes = nullptr;
    if (int rc = X.get(&d_boxes, size_t(n) * 6)) return rc;
    LUX_CUDA(cudaMemcpyAsync(d_boxes, boxes, sizeof(float) * 6 * size_t(n), cudaMemcpyHostToDevice, st));
    DeviceBvh8 b;
    std::vector<int> tb(tree_begin, tree_begin + num_trees + 1);
    if (int rc = build_bvh8_device(d_boxes, tb, 0, false, st, b)) return rc;
    if (b.num_nodes > uint32_t(capacity)) return fail(LUX_ERR_INVALID, "node capacity too small");
    LUX_CUDA(cudaMemcpyAsync(out, b.nodes, sizeof(BVH8Node) * b.num_nodes, cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaMemcpyAsync(order, b.leaf_prim, sizeof(uint32_t) * size_t(n), cudaMemcpyDeviceToHost, st));
    LUX_CUDA(cudaStreamSynchronize(st));
    for (int t = 0; t < num_trees; ++t) {
        roots[t] = b.root[t];
        depth[t] = b.depth[t];
    }
    *num_nodes = int(b.num_nodes);
    return LUX_OK;
}
