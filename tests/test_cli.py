"""The headless command line on the CPU: the reference's flag grammar and messages
(src/main.cpp:81-147), the saveImage pixel rule (src/app/save_image.cpp:42-84) and the PNG
writer. Rendering through it is covered on the GPU in tests/test_gpu_parity.py."""
import os
import tempfile

import numpy as np
import pytest

from luxion_b200 import cli


def test_flags_as_the_reference_parses_them():
    a = cli.parse_args(["scene.glb", "-e", "sky.npy", "-i", "64", "-o", "out/name", "-dmis", "-emis", "-lock"])
    assert a == {"scene": "scene.glb", "envmap": "sky.npy", "iterations": 64, "output": "out/name",
                 "dmis": True, "emis": True, "lock": True, "debug_material": 0, "debug_bvh": False}
    assert cli.parse_args(["s", "--iterations", "3", "--envmap", "e", "--output", "o"])["iterations"] == 3
    assert cli.parse_args(["s"])["iterations"] == 5000          # the reference's default
    for bad, msg in ((["s", "-i"], "requires a number"), (["s", "-i", "0"], "invalid iteration count"),
                     (["s", "-i", "x"], "invalid iteration count"), (["s", "-e"], "requires a path"),
                     (["s", "-o"], "requires a name"), (["a", "b"], "unexpected argument 'b'")):
        with pytest.raises(ValueError, match=msg):
            cli.parse_args(bad)
    with pytest.raises(ValueError):
        cli.parse_args(["-dmis"])
    # the debug views of the reference's ImGui panel (src/app/render_imgui.cpp:336-345)
    assert cli.parse_args(["s", "-debug-material", "3"])["debug_material"] == 3
    assert cli.parse_args(["s", "-debug-bvh"])["debug_bvh"] is True
    for bad, msg in ((["s", "-debug-material"], "requires a number"), (["s", "-debug-material", "7"], "1..6"),
                     (["s", "-debug-material", "1", "-debug-bvh"], "exclusive")):
        with pytest.raises(ValueError, match=msg):
            cli.parse_args(bad)
    assert cli.main([]) == 1
    assert cli.main(["missing.glb"]) == 1    # a scene file that cannot be read


def test_save_image_rule():
    img = np.zeros((2, 3, 3), np.float32)
    img[0, 0] = [2.0, 0.5, 100.0]     # sum over 2 samples
    img[1, 2] = [0.0, 1e-3, 0.2]
    out = cli.to_png_bytes(img, 2)
    def ref(v):
        x = np.float32(v) / np.float32(2)
        a = np.clip((x * (np.float32(2.51) * x + np.float32(0.03))) /
                    (x * (np.float32(2.43) * x + np.float32(0.59)) + np.float32(0.14)), 0, 1).astype(np.float32)
        return int(np.float32(np.clip(np.power(a, np.float32(0.45)), 0, 1)) * np.float32(255))
    # x is mirrored: pixel (x=0) lands in column 2
    assert list(out[0, 2]) == [ref(2.0), ref(0.5), ref(100.0)]
    assert list(out[1, 0]) == [ref(0.0), ref(1e-3), ref(0.2)]
    assert out[0, 2, 2] == 255 and out[1, 0, 0] == 0
    # a material debug view is saved without ACES and gamma, still mirrored
    raw = cli.to_png_bytes(img, 2, tonemap=False)
    assert list(raw[0, 2]) == [255, int(np.float32(0.25) * np.float32(255)), 255]
    assert list(raw[1, 0]) == [0, 0, int(np.float32(0.1) * np.float32(255))]


def test_png_round_trip():
    rng = np.random.default_rng(0)
    rgb = rng.integers(0, 256, (17, 23, 3)).astype(np.uint8)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.png")
        cli.write_png(p, rgb)
        assert np.array_equal(cli.read_png(p), rgb)


def test_envmap_readers_give_rgba():
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")  # before OpenCV is imported
    import cv2
    env = (np.random.default_rng(1).random((6, 10, 3)) * 20).astype(np.float32)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "e.exr")
        assert cv2.imwrite(p, env[..., ::-1])      # OpenCV writes BGR
        got = cli.load_envmap(p)
        assert got.shape == (6, 10, 4) and np.array_equal(got[..., :3], env) and np.all(got[..., 3] == 1)
        q = os.path.join(d, "e.npy")
        np.save(q, env)
        assert np.array_equal(cli.load_envmap(q)[..., :3], env)
