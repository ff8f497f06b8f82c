"""Where the reference's host build (oracle/_ref) is present, the oracle is compared with it on
fresh inputs beyond the golden set: closest-hit distances against the reference's own
meshIntersectionTest, and whole renders in every lighting mode."""
import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.skipif(not ol.ref_available(), reason="reference host build absent")


def scene_rand(seed=3):
    return lx.random_scene(seed=seed, num_instances=10, total_tris=20000, min_tris=1000, max_tris=4000,
                           num_emissive=3, num_textures=4, texture_size=32, env_width=64, env_height=32,
                           width=32, height=24, trace_depth=8)


def test_closest_t_matches_mesh_intersection_test():
    s = scene_rand()
    o, r = ol.OracleScene(s), ol.RefScene(s)
    rays = ol.random_rays(3000, [-12, 0, -12], [12, 5, 12], seed=12)
    # opaque-only comparison: meshIntersectionTest has no alpha test
    hits = o.trace(rays, 0, 1)
    t_ref = r.mesh_isect_t(rays)
    t_orc = hits[:, 0].view(np.float32)
    opaque = np.array([s.desc.materials[s.desc.instances[i].material].alpha_mode == 0 if i != 0xFFFFFFFF else True
                       for i in hits[:, 1]])
    m = opaque & (t_ref > 0)
    assert m.sum() > 100
    assert np.array_equal(t_orc[m], t_ref[m])


@pytest.mark.parametrize("dl,env", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_render_matches_reference(dl, env):
    s = scene_rand(seed=4)
    opt = default_options(direct_light_sampling=dl, env_importance_sampling=env)
    a, sa = ol.OracleScene(s).render(opt, 5, 2)
    b, sb = ol.RefScene(s).render(opt, 5, 2)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(sa, sb)


def test_cornell_render_matches_reference():
    s = lx.cornell36(32, 32)
    opt = default_options(direct_light_sampling=1)
    a, _ = ol.OracleScene(s).render(opt, 1, 3)
    b, _ = ol.RefScene(s).render(opt, 1, 3)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def scene_debug(seed=5):
    """scene_rand with normal maps, metallic-roughness textures and an alpha-blended material,
    so every material debug view has something to show."""
    s = scene_rand(seed=seed)
    d = s.desc
    for k in range(d.num_materials):
        m = d.materials[k]
        if k % 2 == 1:
            m.normal_tex = k % d.num_textures
        if k % 3 == 1:
            m.metallic_roughness_tex = (k + 1) % d.num_textures
        if k == 2:
            m.alpha_mode, m.alpha, m.albedo_tex = 2, 0.6, 0
    return s


@pytest.mark.parametrize("mode", range(1, 7))
def test_material_debug_views_match_reference(mode):
    """render_material_debug_mode (src/material_debug_render.cu:3-26) through the reference's own
    shadePath at trace depth 1 (src/pathtrace.cu:107)."""
    s = scene_debug()
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1, material_debug_mode=mode)
    a, sa = ol.OracleScene(s).render(opt, 3, 2)
    b, sb = ol.RefScene(s).render(opt, 3, 2)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(sa, sb)
    assert sa[2] == 2 * s.width * s.height  # one bounce per sample
