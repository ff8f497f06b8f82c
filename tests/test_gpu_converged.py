"""Converged images against the FP64 CPU integrator (the oracle in double precision) at 4096
samples per pixel. Both sides draw the same per-path random streams, so the relMSE measures
the FP32 arithmetic of each form, not sampling noise: plain FP32 within 1e-4, and the
precision form (FP64 light CDFs, compensated accumulation) within the same bound against the
FP64 integrator built with the same light CDFs and binary16 texels."""
import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200 import _ffi
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.gpu

SPP = 4096
RELMSE_TOL = 1e-4


def relmse(a, b):
    return float(np.mean((a.astype(np.float64) - b) ** 2) / np.mean(b.astype(np.float64) ** 2))


@pytest.fixture(scope="module")
def scene():
    return lx.random_scene(seed=17, num_instances=10, total_tris=20000, min_tris=1000, max_tris=4000, num_emissive=3,
                           num_textures=4, texture_size=32, env_width=64, env_height=32, width=32, height=24,
                           trace_depth=8)


def test_plain_fp32_converges_to_the_fp64_integrator(scene):
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1)
    r = lx.Renderer(scene, opt)
    r.render(1, SPP)
    g = r.image_sum() / SPP
    r.close()
    ref = ol.OracleScene(scene).render(opt, 1, SPP, f64=True)[0] / SPP
    e = relmse(g, ref)
    print("plain FP32 relMSE against FP64 at", SPP, "spp:", e)
    assert e <= RELMSE_TOL


def test_precision_form_converges_to_the_fp64_integrator(scene):
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1, precision=_ffi.PRECISION_COMPENSATED,
                          texture_storage=_ffi.TEXSTORE_HALF)
    r = lx.Renderer(scene, opt)
    r.render(1, SPP)
    g = r.image_sum() / SPP
    r.close()
    ref = ol.OracleScene(scene, cdf_f64=1, tex_storage=_ffi.TEXSTORE_HALF).render(opt, 1, SPP, f64=True)[0] / SPP
    e = relmse(g, ref)
    print("precision form relMSE against FP64 at", SPP, "spp:", e)
    assert e <= RELMSE_TOL
