"""The headless command line end to end on the GPU: the PNG it writes is the saveImage rule
applied to the same render done through the API."""
import os
import tempfile

import numpy as np
import pytest

import luxion_b200 as lx
from luxion_b200 import cli
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.gpu


def test_cli_renders_cornell_with_dmis():
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "cornell")
        assert cli.main(["cornell", "-i", "4", "-o", out, "-dmis", "-lock"]) == 0
        png = cli.read_png(out + ".png")
    r = lx.Renderer(lx.cornell36(256, 256), default_options(direct_light_sampling=1))
    r.render(1, 4)
    want = cli.to_png_bytes(r.image_sum(), 4)
    r.close()
    assert png.shape == (256, 256, 3) and np.array_equal(png, want)


def test_cli_envmap_and_emis():
    env = np.full((16, 32, 3), 0.5, np.float32)
    env[4:6, 10:12] = 50.0
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "sky.npy")
        np.save(p, env)
        out = os.path.join(d, "furn")
        assert cli.main(["furnace", "-e", p, "-i", "2", "-o", out, "-emis"]) == 0
        png = cli.read_png(out + ".png")
    assert png.max() > 0


def test_cli_material_debug_view():
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "albedo")
        assert cli.main(["cornell", "-i", "2", "-o", out, "-dmis", "-debug-material", "1"]) == 0
        png = cli.read_png(out + ".png")
    r = lx.Renderer(lx.cornell36(256, 256), default_options(direct_light_sampling=1, material_debug_mode=1))
    r.render(1, 2)
    img = r.image_sum()
    r.close()
    want = cli.to_png_bytes(img, 2, tonemap=False)
    assert np.array_equal(png, want)
    # the Cornell box's red wall albedo (0.63, 0.065, 0.05) shows as its raw value
    assert (np.abs(want.reshape(-1, 3).astype(int) - [int(np.float32(0.63) * 255), 16, 12]).max(axis=1) <= 1).any()
