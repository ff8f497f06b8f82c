"""A glTF scene through the renderer on the GPU: the scene loaded from a .glb renders in
parity with the oracle on the same description, and the command line renders .glb files."""
import os
import tempfile

import numpy as np
import pytest

import luxion_b200 as lx
import oracle_lib as ol
from luxion_b200 import cli, gltf
from luxion_b200._ffi import default_options

pytestmark = pytest.mark.gpu

ROOM = dict(positions=[[-2, 0, -2], [2, 0, -2], [2, 0, 2], [-2, 0, 2]], indices=[[0, 2, 1], [0, 3, 2]],
            normals=[[0, 1, 0]] * 4, material=0)
LAMP = dict(positions=[[-0.5, 2, -0.5], [0.5, 2, -0.5], [0.5, 2, 0.5], [-0.5, 2, 0.5]], indices=[[0, 1, 2], [0, 2, 3]],
            material=1)
BOX = dict(positions=[[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], indices=[[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]],
           material=None)
MATS = [{"pbrMetallicRoughness": {"baseColorFactor": [0.8, 0.7, 0.6, 1.0], "metallicFactor": 0.0, "roughnessFactor": 0.9}},
        {"pbrMetallicRoughness": {"baseColorFactor": [1, 1, 1, 1], "metallicFactor": 0.0}, "emissiveFactor": [1, 1, 1],
         "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 10.0}}}]
NODES = [{"camera": 0, "translation": [0.0, 1.0, 4.0]}, {"mesh": 0}, {"mesh": 1},
         {"mesh": 2, "translation": [-0.5, 0.0, 0.0], "rotation": [0.0, 0.3826834, 0.0, 0.9238795]}]


def small(sb, w=60, h=40):
    c = sb.camera
    sb.camera = lx.make_camera(w, h, list(c.position), list(c.look_at), c.fov[1])
    return sb


def test_glb_scene_renders_like_the_oracle():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "room.glb")
        gltf.save_glb(p, [ROOM, LAMP, BOX], MATS, NODES, {"aspectRatio": 1.5, "yfov": 0.9})
        sb = small(gltf.load(p))
    opt = default_options(direct_light_sampling=1)
    r = lx.Renderer(sb, opt)
    r.render(1, 8)
    img = r.image_sum()
    r.close()
    ref, _ = ol.OracleScene(sb).render(opt, 1, 8)
    rel = np.abs(img - ref) / np.maximum(np.abs(ref), 1e-6)
    assert img.max() > 0 and np.mean(rel.max(axis=2) < 1e-3) >= 0.999


def test_cli_renders_a_glb_file():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "room.glb")
        gltf.save_glb(p, [ROOM, LAMP, BOX], MATS, NODES, {"aspectRatio": 1.5, "yfov": 0.9})
        out = os.path.join(d, "room")
        assert cli.main([p, "-i", "2", "-o", out, "-dmis"]) == 0
        png = cli.read_png(out + ".png")
    assert png.shape == (1000, 1500, 3) and png.max() > 0
