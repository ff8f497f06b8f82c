"""Parity on the benchmark configurations themselves, through the C-ABI.

C1: the 36-triangle Cornell box, 256x256, 64 spp, trace depth 8, -dmis (the whole image).
C2: the 1M-triangle, 200-instance scene every throughput number is measured on (1920x1080,
    depth 12, -dmis -emis). Its traversal runs the quantised BVH8 boxes, the approximate box
    reciprocals and the slab margin at the depth a large instanced scene reaches, so hits are
    checked bit for bit there: camera rays of a 256x256 centre crop, and the bounce-1 rays of
    those paths in all three trace modes (radiance, DL shadow with tmax, env occlusion).

Tolerances (as in test_gpu_parity.py): hit ids with t/u/v and survivor sets bit-exact;
radiance within 1e-3 relative on >= 99.9 % of pixels and image relMSE <= 1e-4.
"""
import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200 import _ffi
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.gpu

REL_TOL = 1e-3
PIXEL_FRAC = 0.999
RELMSE_TOL = 1e-4


def image_parity(a, b):
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    frac = float(np.mean(rel.max(axis=-1) < REL_TOL))
    relmse = float(np.mean((a - b) ** 2) / max(np.mean(b ** 2), 1e-30))
    return frac, relmse


def test_c1_full_image_parity():
    """C1 in full: 256x256, 64 spp, depth 8, -dmis, against the oracle over the whole image and
    against the reference's own host build on a 64x64 crop."""
    s = lx.cornell36(256, 256)
    assert s.desc.trace_depth == 8
    opt = default_options(direct_light_sampling=1)
    r = lx.Renderer(s, opt)
    r.render(1, 64)
    a = r.image_sum()
    st = r.stats()
    r.close()
    b, sb = ol.OracleScene(s).render(opt, 1, 64)
    frac, relmse = image_parity(a, b)
    assert frac >= PIXEL_FRAC and relmse <= RELMSE_TOL, (frac, relmse)
    assert st["rays_radiance"] == sb[0] and st["rays_shadow"] == sb[1]
    if ol.ref_available():
        crop = (96, 96, 64, 64)
        c, _ = ol.RefScene(s).render(opt, 1, 64, crop=crop)
        frac, relmse = image_parity(a[96:160, 96:160], c)
        assert frac >= PIXEL_FRAC and relmse <= RELMSE_TOL, ("reference crop", frac, relmse)


@pytest.fixture(scope="module", params=[_ffi.BVH_SINGLE_LEVEL, _ffi.BVH_TWO_LEVEL], ids=["single", "two_level"])
def c2(request):
    s = lx.random_scene(seed=0)
    assert s.instanced_tris > 990000 and s.desc.num_instances == 200
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1, bvh_layout=request.param)
    r = lx.Renderer(s, opt)
    o = ol.OracleScene(s)
    W, H = s.width, s.height
    x0, y0 = (W - 256) // 2, (H - 256) // 2
    pix = np.array([(y0 + y) * W + x0 + x for y in range(256) for x in range(256)], np.int32)
    yield s, r, o, opt, pix
    r.close()
    o.close()


def test_c2_camera_hits_bit_exact(c2):
    s, r, o, opt, pix = c2
    rays = ol.camera_paths_to_rays(o.camera_rays(pix, 3))
    hg, ho = r.trace_rays(rays, 0, 3), o.trace(rays, 0, 3)
    assert np.mean(hg[:, 1] != 0xFFFFFFFF) > 0.5
    assert np.array_equal(hg, ho)


def bounce1(o, opt, pix, it):
    """The crop's paths after the camera bounce (oracle shade step on oracle-traced hits), the
    next bounce's light samples and a mask of the live paths."""
    paths = o.camera_rays(pix, it)
    paths[:, 12:18] = o.light_samples(opt, pix, it, 0)
    hits = np.zeros((len(pix), 10), np.uint32)
    hits[:, 0:5] = o.trace(ol.camera_paths_to_rays(paths), 0, it)
    out, surv = o.shade_step(opt, paths, hits, it, 1, 1)
    live = (out[:, 19] == 0) & np.all(np.isfinite(out[:, 0:6]), axis=1)
    nee = o.light_samples(opt, pix, it, 1)
    return paths, hits, out, surv, live, nee


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_c2_bounce1_hits_bit_exact(c2, mode):
    s, r, o, opt, pix = c2
    _, _, out, _, live, nee = bounce1(o, opt, pix, 3)
    assert live.mean() > 0.3
    p = out[live]
    rays = np.zeros((len(p), 8), np.float32)
    rays[:, 0:3] = p[:, 0:3]
    rays[:, 7] = p[:, 18]
    if mode == 0:
        rays[:, 3] = 1e16
        rays[:, 4:7] = p[:, 3:6]
    elif mode == 1:
        # toward the emitter points of the next bounce, tmax = the distance
        d = (nee[live, 0:3] - p[:, 0:3]).astype(np.float32)
        dist = np.sqrt(np.sum(d.astype(np.float64) ** 2, axis=1)).astype(np.float32)
        ok = dist > 1e-3
        rays, d, dist = rays[ok], d[ok], dist[ok]
        rays[:, 4:7] = d / dist[:, None]
        rays[:, 3] = dist
    else:
        rays[:, 3] = 1e16
        rays[:, 4:7] = nee[live, 3:6]
    hg, ho = r.trace_rays(rays, mode, 3), o.trace(rays, mode, 3)
    if mode == 2:
        hg, ho = hg[:, :1], ho[:, :1]
    assert np.array_equal(hg, ho)


def test_c2_shade_step(c2):
    s, r, o, opt, pix = c2
    paths, hits, ref, surv, _, _ = bounce1(o, opt, pix, 3)
    out, surv_g = r.shade_step(paths, hits, 3, 1, 1)
    assert np.array_equal(np.sort(surv_g), np.sort(surv))
    assert np.array_equal(out[:, 19], ref[:, 19])
    for lo, hi in ((0, 3), (3, 6), (6, 9), (9, 12)):
        a, b = out[:, lo:hi], ref[:, lo:hi]
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
        assert np.mean(rel.max(axis=1) < REL_TOL) >= PIXEL_FRAC, (lo, hi)


def test_c2_crop_image_parity(c2):
    """The whole 1080p frame at 4 spp on the GPU; a 64x64 centre crop of it against the oracle."""
    s, r, o, opt, pix = c2
    r.reset()
    r.render(1, 4)
    a = r.image_sum()
    W, H = s.width, s.height
    x0, y0 = (W - 64) // 2, (H - 64) // 2
    b, _ = o.render(opt, 1, 4, crop=(x0, y0, 64, 64))
    frac, relmse = image_parity(a[y0:y0 + 64, x0:x0 + 64], b)
    assert frac >= PIXEL_FRAC and relmse <= RELMSE_TOL, (frac, relmse)


# ---- white furnaces: energy against closed forms ----------------------------------------------
# Lambert-like: base colour 1, metallic 0, ior 1 (the shader clamps it to 1.0001, so the
# dielectric Fresnel and the specular lobe are ~0): expected energy 1, loss below 1e-4.
# GGX: metallic 1, base colour 1 (Schlick F = 1), roughness 1 (alpha 1, D = 1/pi): the
# single-scattering directional albedo is E(mu) = 2 (1 - ln 2) / (1 + mu), mu = n.v, so the
# sphere loses 39 % (grazing) to 69 % (head-on) of the energy, about 25 % of the image mean here.
FURNACES = {"lambert": dict(color=(1, 1, 1), metallic=0.0, roughness=1.0, ior=1.0),
            "ggx": dict(color=(1, 1, 1), metallic=1.0, roughness=1.0)}


@pytest.mark.parametrize("kind", ["lambert", "ggx"])
@pytest.mark.parametrize("emis", [0, 1])
def test_furnace_energy(kind, emis):
    from test_furnace import expected_furnace_image
    W = H = 48
    spp = 256
    s = lx.furnace(W, H, 24, vertex_normals=False, **FURNACES[kind])
    opt = default_options(env_importance_sampling=emis)
    r = lx.Renderer(s, opt)
    r.render(1, spp)
    img = r.image_sum() / np.float32(spp)
    r.close()
    o = ol.OracleScene(s)
    ref = o.render(opt, 1, spp)[0] / np.float32(spp)
    frac, relmse = image_parity(img, ref)
    assert frac >= PIXEL_FRAC and relmse <= RELMSE_TOL, (frac, relmse)
    want = expected_furnace_image(o, s, kind, 64)
    assert abs(float(img.mean()) - float(want.mean())) < 1e-3, (img.mean(), want.mean())


def test_c2_zero_direction_components(c2):
    """Rays with direction components of exactly zero. The C2 camera at (0, 7, 25) looks at
    (0, 1, 0), so view, up and right have exact zeros, and a camera ray whose jittered pixel
    offset rounds to 0 has d.x = 0 (about 3e-5 of the samples of one pixel column). Such a
    component once made the box tests' reciprocal infinite and that axis stop culling, so in the
    single-level layout the ray swept a slab of the whole scene. Hits stay bit-exact (also with
    subnormal components), and the traversal work (lux_trace_rays mode 3: node visits plus
    triangle tests) is that of the same rays with the component at 1e-6 instead."""
    s, r, o, opt, pix = c2
    cam = s.desc.camera
    rng = np.random.default_rng(7)
    n = 2048
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = np.array(cam.position[:], np.float32)
    rays[n // 2:, 0:3] += rng.uniform(-8, 8, (n - n // 2, 3)).astype(np.float32)
    view, up = np.array(cam.view[:], np.float64), np.array(cam.up[:], np.float64)
    py = rng.uniform(-0.5, 0.5, n) * float(cam.height) * float(cam.pixel_length[1])
    d = view[None, :] - up[None, :] * py[:, None]
    d[:, 0] = 0.0
    # a quarter of them along the y or z axis (two zero components)
    k = n // 4
    d[:k] = np.eye(3)[rng.integers(1, 3, k)] * rng.choice([-1.0, 1.0], (k, 1))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 4:7] = d.astype(np.float32)
    rays[:, 3] = 1e16
    rays[:, 7] = np.arange(n, dtype=np.int32).view(np.float32)
    assert np.all(rays[:, 4] == 0.0)
    subnormal = rays.copy()
    subnormal[:, 4] = np.float32(1e-40) * rng.choice([-1.0, 1.0], n).astype(np.float32)
    for case in (rays, subnormal):
        for mode in (0, 2):
            hg, ho = r.trace_rays(case, mode, 2), o.trace(case, mode, 2)
            if mode == 2:
                hg, ho = hg[:, :1], ho[:, :1]
            assert np.array_equal(hg, ho), mode
    w0 = r.trace_rays(rays, 3, 2)
    assert np.array_equal(w0[:, :3], r.trace_rays(rays, 0, 2)[:, :3])
    nudged = rays.copy()
    nudged[:, 4] = np.float32(1e-6)
    w1 = r.trace_rays(nudged, 3, 2)
    work, work_nudged = w0[:, 3].astype(np.float64), w1[:, 3].astype(np.float64)
    assert work.mean() > 5
    assert work.sum() <= 1.25 * work_nudged.sum() + 10 * n, (work.sum(), work_nudged.sum())
    assert work.max() <= 4 * work_nudged.max() + 200, (work.max(), work_nudged.max())
