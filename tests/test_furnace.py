"""White-furnace energy of the shading model, on the CPU oracle, against closed forms.

The sphere is a convex icosphere shaded with its facet normals under a constant environment of
1, so every camera path that hits it scatters once and escapes: the expected pixel value is
the material's directional albedo E(mu) at mu = n.v (1 for a miss).

  * Lambert-like (base colour 1, metallic 0, ior 1 -> clamped to 1.0001 by the shader,
    src/shaders/cook_torrance.cu:80): the dielectric Fresnel is ~0, so k_D = 1 and the
    specular lobe vanishes: E = 1.
  * GGX metal (metallic 1, base colour 1, roughness 1): Schlick F = 1 (cook_torrance.cu:27-31),
    alpha = roughness^2 = 1 gives D = 1/pi (:8-25), and the separable Smith term (:52-67) has
    G1(c) = 2c / (c + 1). Then E(mu) = G1(mu) / (4 pi mu) * int G1(l) dw_l
    = (1 - ln 2) * G1(mu) / mu = 2 (1 - ln 2) / (1 + mu): single scattering loses 39 % of the
    energy at grazing incidence and 69 % head-on.
The oracle, run with and without HDRI importance sampling (-emis, power-heuristic MIS), must
converge to those values within 1e-3 on the image mean.
"""
import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200._ffi import default_options

FURNACES = {"lambert": dict(color=(1, 1, 1), metallic=0.0, roughness=1.0, ior=1.0),
            "ggx": dict(color=(1, 1, 1), metallic=1.0, roughness=1.0)}


def expected_furnace_image(o, s, kind, n_iter):
    """Closed-form expected image of a furnace scene: E(mu) of each camera ray's facet normal,
    averaged over the first n_iter jittered camera iterations (1 where a ray misses)."""
    d = s.desc
    m = d.meshes[0]
    P = np.ctypeslib.as_array(m.positions, shape=(m.num_verts * 3,)).reshape(-1, 3).astype(np.float64)
    idx = np.ctypeslib.as_array(m.indices, shape=(m.num_tris * 3,)).reshape(-1, 3).astype(np.int64)
    fn = np.cross(P[idx[:, 1]] - P[idx[:, 0]], P[idx[:, 2]] - P[idx[:, 0]])
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)
    W, H = s.width, s.height
    pix = np.arange(W * H, dtype=np.int32)
    acc = np.zeros(W * H)
    for it in range(1, n_iter + 1):
        rays = ol.camera_paths_to_rays(o.camera_rays(pix, it))
        h = o.trace(rays, 0, it)
        hit = h[:, 1] != 0xFFFFFFFF
        e = np.ones(W * H)
        if kind == "ggx":
            dd = rays[hit, 4:7].astype(np.float64)
            dd /= np.linalg.norm(dd, axis=1, keepdims=True)
            mu = np.abs(np.einsum("ij,ij->i", dd, fn[h[hit, 2].astype(np.int64)]))
            e[hit] = 2.0 * (1.0 - np.log(2.0)) / (1.0 + mu)
        acc += e
    return (acc / n_iter).reshape(H, W)


@pytest.mark.parametrize("kind", ["lambert", "ggx"])
@pytest.mark.parametrize("emis", [0, 1])
def test_oracle_furnace_energy(kind, emis):
    s = lx.furnace(48, 48, 24, vertex_normals=False, **FURNACES[kind])
    o = ol.OracleScene(s)
    spp = 256
    img = o.render(default_options(env_importance_sampling=emis), 1, spp)[0] / np.float32(spp)
    want = expected_furnace_image(o, s, kind, 64)
    assert abs(float(img.mean()) - float(want.mean())) < 1e-3, (img.mean(), want.mean())
    if kind == "ggx":
        loss = 1.0 - float(want.mean())
        assert 0.2 < loss < 0.3, loss       # the stated single-scattering loss of this view
