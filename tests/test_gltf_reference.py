"""glTF ingestion against the reference's own loader, on the reference's own fixture scenes.

luxion_b200/gltf.py must read scenes/cornell.glb, furnace_test.glb (+ exr/white_furnace.exr),
material_tests.glb and dragon_cornell_box.glb into the same scene description, bit for bit, as
the reference's Scene::loadFromGLTF (src/scene/scene_load_gltf.cpp:61-529, compiled for the host
in oracle/_ref/libluxref_loader.so): meshes, normals, uvs, indices, node matrices and their
glm inverses, materials, textures, camera and environment texels. Those checks need the
reference checkout beside this repository. The committed fixture (tests/golden/
fixture_scenes.npz, the reference loader's output) pins the oracle against the reference's
host build on these scenes everywhere."""
import ctypes as C
import os

import numpy as np
import pytest

import fixture_scenes as fs
import loader_compare as lc
import oracle_lib as ol
from luxion_b200 import cli, gltf
from luxion_b200._ffi import SceneDesc, default_options

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("LUXION_REFERENCE", os.path.normpath(os.path.join(ROOT, "..", "reference")))
LOADER = os.path.join(ROOT, "oracle", "_ref", "libluxref_loader.so")
SCENES = {"cornell": ("cornell.glb", None), "furnace": ("furnace_test.glb", "exr/white_furnace.exr"),
          "material_tests": ("material_tests.glb", None), "dragon": ("dragon_cornell_box.glb", None)}
need_ref = pytest.mark.skipif(not (os.path.isdir(os.path.join(REF, "scenes")) and os.path.exists(LOADER)),
                              reason="reference checkout or its host loader build absent")


def ref_loader():
    L = C.CDLL(LOADER)
    L.ref_load_gltf.restype = C.c_void_p
    L.ref_load_gltf.argtypes = [C.c_char_p, C.c_char_p]
    L.ref_loaded_desc.restype = C.POINTER(SceneDesc)
    L.ref_loaded_desc.argtypes = [C.c_void_p]
    L.ref_loaded_free.argtypes = [C.c_void_p]
    return L


def ours(tag):
    glb, exr = SCENES[tag]
    sb = gltf.load(os.path.join(REF, "scenes", glb))
    if exr:
        sb.set_env(cli.load_envmap(os.path.join(REF, "scenes", exr)))
    return sb


@need_ref
@pytest.mark.parametrize("tag", list(SCENES))
def test_loader_matches_reference_loader(tag):
    glb, exr = SCENES[tag]
    L = ref_loader()
    h = L.ref_load_gltf(os.path.join(REF, "scenes", glb).encode(),
                        os.path.join(REF, "scenes", exr).encode() if exr else None)
    try:
        sb = ours(tag)
        assert lc.compare_descs(sb.desc_ptr.contents, L.ref_loaded_desc(h).contents) == []
    finally:
        L.ref_loaded_free(h)


@need_ref
@pytest.mark.parametrize("tag", fs.TAGS)
def test_committed_fixture_is_the_loaded_scene(tag):
    assert lc.compare_descs(ours(tag).desc_ptr.contents, fs.fixture_scene(tag).desc_ptr.contents) == []


def fixture_options(tag):
    """cornell: NEE on its ceiling light (-dmis); furnace: HDRI sampling of the white furnace
    (-emis); material_tests has no light of its own and renders under a synthetic sky (-emis)."""
    return default_options(direct_light_sampling=1 if tag == "cornell" else 0,
                           env_importance_sampling=0 if tag == "cornell" else 1)


def lit_fixture(tag):
    s = fs.fixture_scene(tag)
    if tag == "material_tests":
        h, w = 64, 128
        y = (np.arange(h, dtype=np.float32) + 0.5) / h
        sky = np.zeros((h, w, 4), np.float32)
        sky[..., 0] = (0.4 + 1.6 * (1 - y))[:, None]
        sky[..., 1] = (0.5 + 1.4 * (1 - y))[:, None]
        sky[..., 2] = (0.7 + 1.2 * (1 - y))[:, None]
        sky[..., 3] = 1.0
        sky[4:8, 20:26, :3] = 60.0  # a small sun
        s.set_env(sky)
    return s


@pytest.mark.skipif(not ol.ref_available(), reason="reference host build absent")
@pytest.mark.parametrize("tag", fs.TAGS)
def test_oracle_matches_reference_build_on_fixture_scenes(tag):
    s = lit_fixture(tag)
    opt = fixture_options(tag)
    crop = ((s.width - 48) // 2, (s.height - 48) // 2, 48, 48)
    a, sa = ol.OracleScene(s).render(opt, 1, 8, crop=crop)
    b, sb = ol.RefScene(s).render(opt, 1, 8, crop=crop)
    assert b.mean() > 0
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    assert np.mean(rel.max(axis=-1) < 1e-3) >= 0.999
    assert np.mean((a - b) ** 2) / np.mean(b ** 2) <= 1e-4
