"""Measure the hardware bilinear filter of the GPU (run on a B200):

    python tests/golden/probe_texture_filter.py

Textures whose texel (i, j) holds 1 in channel (i % 2) + 2 * (j % 2) and 0 elsewhere make
every fetch return its four 2-D filter weights, one per channel. The script samples them at
random and at grid coordinates on textures of several sizes, plus an 8-bit ramp for the
unorm path and random texels stored as binary16, and stores every fourth sample, with the weights as integers in units of 1/256,
in texture_filter_probe.npz. The oracle's texture fetch (oracle/lux_oracle.cpp, tex_axis and
tex_fetch) restates the rule these data pin, and tests/test_texture_model.py checks it against
them on the CPU. `--compact-from RAW.npz` rewrites a full-size measurement (PROBE_RAW=1 keeps
all samples) into that committed form.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import luxion_b200 as lx  # noqa: E402
from luxion_b200 import _ffi  # noqa: E402
from luxion_b200.scene_builder import SceneBuilder  # noqa: E402

SIZES = [(54, 38), (1000, 500), (2048, 1024), (6, 4)]


def parity_texture(w, h):
    t = np.zeros((h, w, 4), np.float32)
    j, i = np.mgrid[0:h, 0:w]
    t[j, i, (i % 2) + 2 * (j % 2)] = 1.0
    return t


def main():
    sb = SceneBuilder(8, 8)
    m = sb.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0]], [[0, 1, 2]])
    sb.add_instance(m, sb.add_material())
    ids = [sb.add_texture(parity_texture(w, h), _ffi.TEX_RGBA32F) for (w, h) in SIZES]
    ramp = np.zeros((6, 254, 4), np.uint8)
    ramp[..., 0] = np.arange(254)[None, :]
    ramp[..., 1] = 253 - np.arange(254)[None, :]
    ramp[..., 2] = (np.arange(6) * 50)[:, None]
    ramp[..., 3] = 255
    t_ramp = sb.add_texture(ramp, _ffi.TEX_RGBA8)
    sb.set_env(np.ones((4, 8, 4), np.float32))
    r = lx.Renderer(sb, lx.default_options(texture_storage=_ffi.TEXSTORE_UNORM8))
    rng = np.random.default_rng(1234)
    out = {"sizes": np.array(SIZES, np.int32)}
    for k, (w, h) in enumerate(SIZES):
        uv = np.concatenate([rng.uniform(-3, 3, (30000, 2)), rng.uniform(0, 1, (30000, 2)),
                             rng.uniform(-1e-3, 1e-3, (2000, 2)) + rng.integers(0, 4, (2000, 2)) / np.array([w, h])]
                            ).astype(np.float32)
        out[f"uv_{k}"] = uv
        out[f"w_{k}"] = r.sample_texture(ids[k], uv)
    uv = np.stack([rng.uniform(-2, 2, 30000), rng.uniform(-2, 2, 30000)], 1).astype(np.float32)
    out["uv_ramp"] = uv
    out["ramp"] = ramp
    out["v_ramp"] = r.sample_texture(t_ramp, uv)
    r.close()
    # binary16 storage: random texels (uniform, 8-bit, and over six decades) filtered from half
    sb = SceneBuilder(8, 8)
    m = sb.add_mesh([[-1, -1, 0], [1, -1, 0], [1, 1, 0]], [[0, 1, 2]])
    sb.add_instance(m, sb.add_material())
    half_src = [rng.uniform(0, 100, (16, 24, 4)).astype(np.float32),
                rng.integers(0, 256, (37, 53, 4)).astype(np.uint8),
                np.exp(rng.uniform(np.log(1e-3), np.log(1e3), (32, 64, 4))).astype(np.float32)]
    hids = [sb.add_texture(t, _ffi.TEX_RGBA8 if t.dtype == np.uint8 else _ffi.TEX_RGBA32F) for t in half_src]
    sb.set_env(np.ones((4, 8, 4), np.float32))
    r = lx.Renderer(sb, lx.default_options(texture_storage=_ffi.TEXSTORE_HALF))
    for k, (t, tid) in enumerate(zip(half_src, hids)):
        f = t.astype(np.float32) / np.float32(255) if t.dtype == np.uint8 else t
        out[f"half_tex_{k}"] = f.astype(np.float16)
        uv = rng.uniform(-3, 3, (6000, 2)).astype(np.float32)
        out[f"half_uv_{k}"] = uv
        out[f"half_v_{k}"] = r.sample_texture(tid, uv)
    r.close()
    dst = os.environ.get("PROBE_OUT", os.path.join(HERE, "texture_filter_probe.npz"))
    np.savez_compressed(dst, **(out if os.environ.get("PROBE_RAW") else compact(out)))
    print("wrote", dst)


def compact(raw):
    """Every fourth sample; parity-texture weights as exact integers (x256, uint16)."""
    out = {"sizes": raw["sizes"], "ramp": raw["ramp"]}
    for k in range(len(raw["sizes"])):
        out[f"uv_{k}"] = raw[f"uv_{k}"][::4]
        w = raw[f"w_{k}"][::4].astype(np.float64) * 256.0
        assert np.array_equal(w, np.rint(w))
        out[f"w_{k}"] = w.astype(np.uint16)
    out["uv_ramp"] = raw["uv_ramp"][::4]
    out["v_ramp"] = raw["v_ramp"][::4]
    for k in ("half_tex", "half_uv", "half_v"):
        for i in range(3):
            if f"{k}_{i}" in raw:
                out[f"{k}_{i}"] = raw[f"{k}_{i}"]
    return out


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--compact-from":
        raw = dict(np.load(sys.argv[2]))
        np.savez_compressed(os.path.join(HERE, "texture_filter_probe.npz"), **compact(raw))
        print("wrote", os.path.join(HERE, "texture_filter_probe.npz"))
    else:
        main()
