"""Write tests/golden/fixture_scenes.npz: the reference's own fixture scenes as its own loader
reads them.

    python tests/golden/make_fixture_scenes.py [REFERENCE_TREE]

The scenes scenes/cornell.glb, scenes/furnace_test.glb with scenes/exr/white_furnace.exr and
scenes/material_tests.glb of the reference tree are loaded by the reference's Scene::loadFromGLTF
(src/scene/scene_load_gltf.cpp:61-529), compiled for the host (oracle/_ref/libluxref_loader.so,
built by oracle/Makefile), and stored field for field: per mesh its positions, normals, uvs and
indices; per instance its mesh, material and the three matrices; the materials and the camera
as the C-ABI structs' bytes; the trace depth; the float texels of textures and environment map.
tests/fixture_scenes.py turns a stored scene back into a scene description. The reference tree
defaults to the checkout beside this repository. dragon_cornell_box.glb (14 MB, 600k triangles)
is left out for its size; tests/test_gltf_reference.py checks it where the reference tree is.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from luxion_b200._ffi import CameraDesc, MaterialDesc, SceneDesc  # noqa: E402

OUT = os.path.join(HERE, "fixture_scenes.npz")
SCENES = (("cornell", "cornell.glb", None), ("furnace", "furnace_test.glb", "exr/white_furnace.exr"),
          ("material_tests", "material_tests.glb", None))
LOADER_SO = os.path.join(ROOT, "oracle", "_ref", "libluxref_loader.so")


def reference_loader():
    L = C.CDLL(LOADER_SO)
    L.ref_load_gltf.restype = C.c_void_p
    L.ref_load_gltf.argtypes = [C.c_char_p, C.c_char_p]
    L.ref_loaded_desc.restype = C.POINTER(SceneDesc)
    L.ref_loaded_desc.argtypes = [C.c_void_p]
    L.ref_loaded_free.argtypes = [C.c_void_p]
    return L


def store(tag, d, out):
    for m in range(d.num_meshes):
        md = d.meshes[m]
        out[f"{tag}_mesh{m}_pos"] = np.ctypeslib.as_array(md.positions, shape=(md.num_verts, 3)).copy()
        out[f"{tag}_mesh{m}_idx"] = np.ctypeslib.as_array(md.indices, shape=(md.num_tris, 3)).copy()
        if md.normals:
            out[f"{tag}_mesh{m}_nrm"] = np.ctypeslib.as_array(md.normals, shape=(md.num_verts, 3)).copy()
        if md.uvs:
            out[f"{tag}_mesh{m}_uv"] = np.ctypeslib.as_array(md.uvs, shape=(md.num_verts, 2)).copy()
    n = d.num_instances
    out[f"{tag}_inst_mesh"] = np.array([d.instances[i].mesh for i in range(n)], np.int32)
    out[f"{tag}_inst_mat"] = np.array([d.instances[i].material for i in range(n)], np.int32)
    out[f"{tag}_inst_xf"] = np.array([[list(d.instances[i].transform), list(d.instances[i].inverse),
                                       list(d.instances[i].inv_transpose)] for i in range(n)], np.float32)
    out[f"{tag}_mats"] = np.frombuffer(bytes((MaterialDesc * d.num_materials).from_address(
        C.addressof(d.materials.contents))), np.uint8).copy()
    out[f"{tag}_camera"] = np.frombuffer(bytes(CameraDesc.from_buffer_copy(d.camera)), np.uint8).copy()
    out[f"{tag}_trace_depth"] = np.array([d.trace_depth], np.int32)
    for t in range(d.num_textures):
        x = d.textures[t]
        out[f"{tag}_tex{t}"] = np.ctypeslib.as_array(C.cast(x.data, C.POINTER(C.c_float)),
                                                     shape=(x.height, x.width, 4)).copy()
    if d.env_data:
        out[f"{tag}_env"] = np.ctypeslib.as_array(C.cast(d.env_data, C.POINTER(C.c_float)),
                                                  shape=(d.env_height, d.env_width, 4)).copy()


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.path.normpath(os.path.join(ROOT, "..", "reference"))
    if not os.path.exists(LOADER_SO):
        raise SystemExit("oracle/_ref/libluxref_loader.so is missing: build it with `make -C oracle` where the "
                         "reference tree is present")
    L = reference_loader()
    out = {}
    for tag, glb, exr in SCENES:
        h = L.ref_load_gltf(os.path.join(ref, "scenes", glb).encode(),
                            os.path.join(ref, "scenes", exr).encode() if exr else None)
        store(tag, L.ref_loaded_desc(h).contents, out)
        L.ref_loaded_free(h)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
