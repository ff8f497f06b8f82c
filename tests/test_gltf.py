"""The glTF loader (luxion_b200.gltf) on the CPU: a .glb written by the tests' own writer loads
into the scene the reference's loader would build (src/scene/scene_load_gltf.cpp:61-529):
default red material first, glTF material fields and extensions, node transforms composed down
the hierarchy, normalised normals, the camera of the camera node at a 1000-pixel short side."""
import math
import os
import tempfile

import numpy as np
import pytest

from luxion_b200 import _ffi, gltf

QUAD = dict(positions=[[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], indices=[[0, 1, 2], [0, 2, 3]],
            normals=[[0, 0, 2], [0, 0, 2], [0, 0, 3], [0, 0, 1]], uvs=[[0, 0], [1, 0], [1, 1], [0, 1]], material=1)
TET = dict(positions=[[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], indices=[[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]],
           material=None)
MATERIALS = [
    {"pbrMetallicRoughness": {"baseColorFactor": [0.2, 0.4, 0.6, 0.8], "metallicFactor": 0.3,
                              "roughnessFactor": 0.7}},
    {"pbrMetallicRoughness": {"baseColorTexture": {"index": 0, "extensions": {"KHR_texture_transform": {
        "offset": [0.25, 0.5], "scale": [2.0, 3.0], "rotation": 0.5}}}},
     "emissiveFactor": [1.0, 0.5, 0.25], "alphaMode": "MASK", "alphaCutoff": 0.3,
     "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 4.0}, "KHR_materials_ior": {"ior": 1.33},
                    "KHR_materials_transmission": {"transmissionFactor": 0.9}}},
]
ROT = [0.0, math.sin(0.25), 0.0, math.cos(0.25)]          # 0.5 rad about +y
NODES = [
    {"camera": 0, "translation": [0.0, 1.0, 5.0]},
    {"mesh": 0, "translation": [1.0, 2.0, 3.0], "rotation": ROT, "scale": [2.0, 2.0, 2.0], "children": [2]},
    {"mesh": 1, "matrix": [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0.5, 0, 0, 1]},
]


def write(path):
    tex = np.zeros((4, 4, 4), np.uint8)
    tex[..., 0] = 200
    tex[..., 3] = np.arange(16, dtype=np.uint8).reshape(4, 4) * 16
    gltf.save_glb(path, [QUAD, TET], MATERIALS, NODES, {"aspectRatio": 1.5, "yfov": 0.8, "znear": 0.1},
                  images=[tex])
    return tex


@pytest.fixture(scope="module")
def loaded():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "t.glb")
        tex = write(p)
        yield gltf.load(p), tex


def quat(x, y, z, w):
    """Rotation matrix of the unit quaternion (x, y, z, w), in double (row-major)."""
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y), 0],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x), 0],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y), 0],
                     [0, 0, 0, 1]], np.float64)


def test_materials(loaded):
    sb, _ = loaded
    assert len(sb.materials) == 3
    red = sb.materials[0]
    assert list(red.color) == [1.0, 0.0, 0.0] and red.roughness == 0.0 and red.metallic == 0.0
    m1 = sb.materials[1]
    assert np.allclose(list(m1.color), [0.2, 0.4, 0.6]) and abs(m1.alpha - 0.8) < 1e-7
    assert abs(m1.metallic - 0.3) < 1e-7 and abs(m1.roughness - 0.7) < 1e-7 and abs(m1.ior - 1.55) < 1e-7
    assert m1.albedo_tex == -1 and m1.alpha_mode == _ffi.ALPHA_OPAQUE and m1.emission_strength == 1.0
    m2 = sb.materials[2]
    assert m2.metallic == 1.0 and m2.roughness == 1.0                     # glTF defaults
    assert m2.albedo_tex == 0 and m2.alpha_mode == _ffi.ALPHA_MASK and abs(m2.alpha_cutoff - 0.3) < 1e-7
    assert m2.emission_strength == 4.0 and list(m2.emission_color) == [1.0, 0.5, 0.25]
    assert abs(m2.ior - 1.33) < 1e-7 and abs(m2.transmission - 0.9) < 1e-7
    assert list(m2.albedo_tt.offset) == [0.25, 0.5] and list(m2.albedo_tt.scale) == [2.0, 3.0]
    assert m2.albedo_tt.rotation == 0.5


def test_texture(loaded):
    sb, tex = loaded
    assert len(sb.textures) == 1
    t = sb.textures[0]
    assert (t.width, t.height, t.format) == (4, 4, _ffi.TEX_RGBA8)
    got = np.ctypeslib.as_array((np.ctypeslib.ctypes.c_uint8 * 64).from_address(t.data)).reshape(4, 4, 4)
    assert np.array_equal(got, tex)


def test_instances_and_transforms(loaded):
    sb, _ = loaded
    assert len(sb.instances) == 2 and len(sb.meshes) == 2
    T = np.eye(4)
    T[:3, 3] = [1, 2, 3]
    G1 = T @ quat(*ROT) @ np.diag([2.0, 2.0, 2.0, 1.0])
    G2 = G1 @ np.array([[1, 0, 0, 0.5], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], np.float64)
    for inst, G, mat in zip(sb.instances, (G1, G2), (2, 0)):
        M = np.array(inst.transform[:], np.float32).reshape(4, 4).T        # stored column-major
        assert np.allclose(M, G, atol=1e-6)
        assert inst.material == mat                                         # no material: the red default
    q = sb.meshes[0]
    n = np.ctypeslib.as_array(q.normals, shape=(4, 3))
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-6) and q.num_tris == 2
    assert not sb.meshes[1].normals and not sb.meshes[1].uvs and sb.meshes[1].num_tris == 4


def test_camera(loaded):
    sb, _ = loaded
    c = sb.camera
    assert (c.width, c.height) == (1500, 1000) and sb.trace_depth == 8
    assert list(c.position) == [0.0, 1.0, 5.0] and list(c.view) == [0.0, 0.0, -1.0]
    assert list(c.right) == [1.0, 0.0, 0.0] and list(c.up) == [0.0, 1.0, 0.0]
    y = math.tan(0.5 * math.degrees(0.8) * math.pi / 180)
    assert abs(c.pixel_length[1] - 2 * y / 1000) < 1e-7 and abs(c.pixel_length[0] - 2 * y * 1.5 / 1500) < 1e-7


def test_errors():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "nocam.glb")
        gltf.save_glb(p, [TET], [], [{"mesh": 0}], {"aspectRatio": 1.0, "yfov": 0.8})
        with pytest.raises(gltf.GltfError, match="no camera"):
            gltf.load(p)
