"""The oracle's texture filter against the B200 hardware filter, on the CPU.

tests/golden/texture_filter_probe.npz holds what tests/golden/probe_texture_filter.py read back
from the GPU's bilinear, wrap-mode, normalized-coordinate fetch: the four 2-D weights of
random and near-boundary coordinates on textures of several sizes (power-of-two and not), and
8-bit ramp texels through the unorm path. The oracle must give the same answers bit for bit.
The reference samples its textures with the same hardware fetch (tex2D on a cudaTextureObject
created with linear filtering and wrap addressing: texture.cpp, shade_path.cu tex2D<float4>
calls), so pinning the oracle to the hardware pins it to the reference.
"""
import os

import numpy as np

import oracle_lib as ol
from luxion_b200 import _ffi
from luxion_b200.scene_builder import SceneBuilder

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE = np.load(os.path.join(HERE, "golden", "texture_filter_probe.npz"))


def parity_texture(w, h):
    t = np.zeros((h, w, 4), np.float32)
    j, i = np.mgrid[0:h, 0:w]
    t[j, i, (i % 2) + 2 * (j % 2)] = 1.0
    return t


def _scene(storage):
    sb = SceneBuilder(8, 8)
    m = sb.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0]], [[0, 1, 2]])
    sb.add_instance(m, sb.add_material())
    ids = [sb.add_texture(parity_texture(int(w), int(h)), _ffi.TEX_RGBA32F) for (w, h) in PROBE["sizes"]]
    t_ramp = sb.add_texture(PROBE["ramp"], _ffi.TEX_RGBA8)
    sb.set_env(np.ones((4, 8, 4), np.float32))
    return ol.OracleScene(sb, tex_storage=storage), ids, t_ramp


def test_weights_match_hardware_on_every_size():
    o, ids, _ = _scene(_ffi.TEXSTORE_FLOAT)
    for k, tex in enumerate(ids):
        got = o.sample_texture(tex, PROBE[f"uv_{k}"]).astype(np.float64) * 256.0
        want = PROBE[f"w_{k}"].astype(np.float64)
        assert np.array_equal(got, want), (tuple(PROBE["sizes"][k]), int((got != want).any(axis=1).sum()))


def test_unorm8_path_matches_hardware():
    o, _, t_ramp = _scene(_ffi.TEXSTORE_UNORM8)
    got = o.sample_texture(t_ramp, PROBE["uv_ramp"])
    assert np.array_equal(got.view(np.uint32), PROBE["v_ramp"].view(np.uint32))


def test_a_plain_float_product_model_would_not_match():
    """The measured coordinate rule matters: the single-precision u * n - 0.5 form misses some
    weights on non-power-of-two sizes. This is the check that the fixture can tell rules apart."""
    k = 1  # 1000 x 500
    w, h = (int(x) for x in PROBE["sizes"][k])
    uv = PROBE[f"uv_{k}"]
    u = uv[:, 0] - np.floor(uv[:, 0])
    x = (u * np.float32(w)).astype(np.float32) - np.float32(0.5)
    a_fp32 = np.floor((x - np.floor(x)) * np.float32(256) + np.float32(0.5))
    wt = PROBE[f"w_{k}"].astype(np.int64)
    i0 = np.floor(x).astype(np.int64) % 2
    a_meas = np.where(i0 == 0, wt[:, 1] + wt[:, 3], wt[:, 0] + wt[:, 2])
    assert (a_meas != a_fp32).sum() > 50


def test_binary16_filter_matches_hardware():
    """Texels held as binary16 (the precision form's storage, and any RGBA16F input) take the
    hardware's half filter: block-aligned 15-bit texels, exact sum, ties away from zero."""
    sb = SceneBuilder(8, 8)
    m = sb.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0]], [[0, 1, 2]])
    sb.add_instance(m, sb.add_material())
    ids = [sb.add_texture(PROBE[f"half_tex_{k}"], _ffi.TEX_RGBA16F) for k in range(3)]
    sb.set_env(np.ones((4, 8, 4), np.float32))
    o = ol.OracleScene(sb, tex_storage=_ffi.TEXSTORE_FLOAT)
    for k, tex in enumerate(ids):
        got = o.sample_texture(tex, PROBE[f"half_uv_{k}"])
        want = PROBE[f"half_v_{k}"]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (k, int((got != want).sum()))


def test_binary16_storage_rounds_then_filters_as_half():
    """Float input under LUX_TEXSTORE_HALF: texels round to nearest-even binary16 first."""
    tex = PROBE["half_tex_0"]
    sb = SceneBuilder(8, 8)
    m = sb.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0]], [[0, 1, 2]])
    sb.add_instance(m, sb.add_material())
    t_half = sb.add_texture(tex, _ffi.TEX_RGBA16F)
    # the same texels given as float32 with a residue below half precision
    t_f32 = sb.add_texture(tex.astype(np.float32) * np.float32(1 + 2 ** -13), _ffi.TEX_RGBA32F)
    sb.set_env(np.ones((4, 8, 4), np.float32))
    o = ol.OracleScene(sb, tex_storage=_ffi.TEXSTORE_HALF)
    uv = PROBE["half_uv_0"]
    assert np.array_equal(o.sample_texture(t_half, uv), o.sample_texture(t_f32, uv))
