"""Generate the golden vectors of the render path from the reference's own sources.

    python tests/golden/make_golden.py

The reference (seabiscuit-iv/luxion) ships no tests and no golden data, so the vectors are
produced by its own hot-path sources compiled for the host (oracle/_ref/libluxref.so, built
by oracle/Makefile from the reference tree in place). Inputs are the seeded procedural
scenes of this repository and seeded random arrays; outputs are stored bit for bit. The
oracle restatement (oracle/lux_oracle.cpp) and the CUDA path are then checked against these
files, so the checks also run where the reference tree is absent.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import luxion_b200 as lx  # noqa: E402
import oracle_lib as ol  # noqa: E402
from luxion_b200._ffi import default_options  # noqa: E402

OUT = os.path.join(HERE, "golden.npz")


def small_random_scene():
    """The small textured scene of the golden set (HDRI, alpha masks, transmission)."""
    return lx.random_scene(seed=7, num_instances=8, total_tris=16000, min_tris=1000, max_tris=4000, num_emissive=2,
                           num_textures=4, texture_size=64, env_width=128, env_height=64, width=40, height=32,
                           trace_depth=6)


def bsdf_records(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)

    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    rec = np.zeros((n, 16), np.float32)
    rec[:, 0:3] = unit(n)          # wo
    rec[:, 3:6] = unit(n)          # n
    rec[:, 6:9] = unit(n)          # wi
    rec[:, 9:12] = rng.uniform(0.0, 1.0, (n, 3))
    rec[:, 12] = rng.uniform(0.0, 1.0, n)
    rec[:, 13] = (rng.uniform(size=n) < 0.3).astype(np.float32)
    rec[:, 14] = rng.uniform(1.0, 2.0, n)
    rec[:, 15] = (rng.uniform(size=n) < 0.2).astype(np.float32)
    return rec


def shade_inputs(scene_oracle, opt, pixels, it):
    """Camera paths of the given pixels plus their traced hits (10 words per path)."""
    paths = scene_oracle.camera_rays(pixels, it)
    paths[:, 12:18] = scene_oracle.light_samples(opt, pixels, it, 0)
    rays = ol.camera_paths_to_rays(paths)
    hits = np.zeros((len(pixels), 10), np.uint32)
    hits[:, 0:5] = scene_oracle.trace(rays, 0, it)
    return paths, hits


def main():
    import ctypes as C
    if not ol.ref_available():
        raise SystemExit("oracle/_ref/libluxref.so is missing: build it with `make -C oracle` where the "
                         "reference tree is present")
    R = ol.ref()
    g = {}
    # RNG streams
    seeds = np.array([(1, 0, 0), (3, 1234, 5), (64, 65535, 8), (1, 2073599, 12), (1000, 77, 1), (2, 1, 31)], np.int32)
    g["rng_seeds"] = seeds
    st = np.zeros((len(seeds), 32), np.float32)
    for i, (a, b, c) in enumerate(seeds):
        R.ref_rng_stream(int(a), int(b), int(c), 32, ol.f32p(st[i]))
    g["rng_streams"] = st
    hv = np.array([0, 1, 2, 0xFFFFFFFF, 123456789, 0x80000000, 0x7FFFFFFF], np.uint32)
    g["hash_in"] = hv
    g["hash_out"] = np.array([R.ref_utilhash(int(x)) for x in hv], np.uint32)
    # CDF search
    rng = np.random.default_rng(3)
    cdf = np.cumsum(rng.uniform(0, 1, 97)).astype(np.float32)
    cdf /= cdf[-1]
    cdf[-1] = 1.0
    xs = np.concatenate([rng.uniform(0, 1, 500), cdf[:20], [0.0, 1.0]]).astype(np.float32)
    g["cdf"] = cdf
    g["cdf_xi"] = xs
    g["cdf_idx"] = np.array([R.ref_select_from_cdf(ol.f32p(cdf), len(cdf), C.c_float(float(x))) for x in xs], np.int32)
    # uber-shader evaluation and sampling
    rec = bsdf_records(3000, 11)
    out = np.zeros((len(rec), 16), np.float32)
    R.ref_eval_bsdf(ol.f32p(rec), len(rec), ol.f32p(out))
    g["bsdf_in"], g["bsdf_out"] = rec, out
    sseeds = np.stack([rng.integers(1, 100, 3000), rng.integers(0, 1 << 21, 3000), rng.integers(0, 13, 3000)], 1).astype(np.int32)
    sout = np.zeros((3000, 4), np.float32)
    R.ref_sample_bsdf(ol.f32p(rec), ol.i32p(sseeds), 3000, ol.f32p(sout))
    g["sample_seeds"], g["sample_out"] = sseeds, sout
    nrm = rec[:1000, 3:6].copy()
    hout = np.zeros((1000, 3), np.float32)
    R.ref_hemisphere(ol.f32p(nrm), ol.i32p(sseeds[:1000]), 1000, ol.f32p(hout))
    g["hemi_n"], g["hemi_out"] = nrm, hout
    # scenes
    for tag, scene, opt in (("cornell", lx.cornell36(48, 48), default_options(direct_light_sampling=1)),
                            ("rand", small_random_scene(),
                             default_options(direct_light_sampling=1, env_importance_sampling=1))):
        rs = ol.RefScene(scene)
        os_ = ol.OracleScene(scene)
        cd = rs.cdfs()
        for k, v in cd.items():
            g[f"{tag}_cdf_{k}"] = np.asarray(v, np.float32)
        npix = scene.width * scene.height
        pix = np.arange(npix, dtype=np.int32)
        cam = rs.camera_rays(pix, 3)
        g[f"{tag}_camera_it3"] = cam
        for depth in (0, 1, 4):
            g[f"{tag}_light_d{depth}"] = rs.light_samples(opt, pix, 3, depth)
        rays = ol.camera_paths_to_rays(cam)
        g[f"{tag}_trace_cam"] = rs.trace(rays, 0, 3)
        lo, hi = ([-0.9, 0.1, -0.9], [0.9, 1.9, 0.9]) if tag == "cornell" else ([-12, 0, -12], [12, 5, 12])
        rr = ol.random_rays(4000, lo, hi, seed=5)
        g[f"{tag}_rand_rays"] = rr
        g[f"{tag}_trace_rand_m0"] = rs.trace(rr, 0, 3)
        g[f"{tag}_trace_rand_m2"] = rs.trace(rr, 2, 3)
        rr1 = rr.copy()
        rr1[:, 3] = np.random.default_rng(9).uniform(0.05, 6.0, len(rr1)).astype(np.float32)
        g[f"{tag}_rand_rays_tmax"] = rr1
        g[f"{tag}_trace_rand_m1"] = rs.trace(rr1, 1, 3)
        # one shade step from the camera, inputs produced by the oracle (pinned above)
        paths, hits = shade_inputs(os_, opt, pix, 3)
        if tag == "rand":
            sh_rays = np.zeros((npix, 8), np.float32)  # env occlusion rays are traced inside the drivers
        out_paths, surv = rs.shade_step(opt, paths, hits, 3, 1, 1)
        g[f"{tag}_shade_in_paths"], g[f"{tag}_shade_in_hits"] = paths, hits
        g[f"{tag}_shade_out_paths"], g[f"{tag}_shade_survivors"] = out_paths, np.sort(surv)
        # small render
        img, stats = rs.render(opt, 1, 2)
        g[f"{tag}_render_2spp"] = img
        g[f"{tag}_render_stats"] = stats
        # Morton keys with the Morton box of the first instance
        m0 = scene.desc.meshes[scene.desc.instances[0].mesh]
        pos = np.ctypeslib.as_array(m0.positions, shape=(m0.num_verts * 3,)).reshape(-1, 3)
        bmin = (pos.min(0).astype(np.float32) - np.float32(1e-5)).astype(np.float32)
        bmax = (pos.max(0).astype(np.float32) + np.float32(1e-5)).astype(np.float32)
        g[f"{tag}_morton"] = rs.morton(rr, bmin, bmax)
    np.savez_compressed(OUT, **g)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
