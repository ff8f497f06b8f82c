"""The reference's fixture scenes (cornell, furnace_test with white_furnace.exr, material_tests)
as its own loader reads them, rebuilt from tests/golden/fixture_scenes.npz (written by
tests/golden/make_fixture_scenes.py) into scene descriptions. Test infrastructure."""
import ctypes
import os

import numpy as np

from luxion_b200 import _ffi
from luxion_b200._ffi import CameraDesc, MaterialDesc
from luxion_b200.scene_builder import SceneBuilder

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fixture_scenes.npz")
TAGS = ("cornell", "furnace", "material_tests")


def fixture_scene(tag: str, g=None) -> SceneBuilder:
    g = np.load(FIXTURES) if g is None else g
    sb = SceneBuilder()
    m = 0
    while f"{tag}_mesh{m}_pos" in g:
        k = f"{tag}_mesh{m}_"
        sb.add_mesh(g[k + "pos"], g[k + "idx"], normals=g[k + "nrm"] if k + "nrm" in g else None,
                    uvs=g[k + "uv"] if k + "uv" in g else None)
        m += 1
    mats = g[f"{tag}_mats"]
    size = ctypes.sizeof(MaterialDesc)
    for i in range(len(mats) // size):
        sb.add_material(MaterialDesc.from_buffer_copy(mats[i * size:(i + 1) * size].tobytes()))
    t = 0
    while f"{tag}_tex{t}" in g:
        sb.add_texture(g[f"{tag}_tex{t}"], _ffi.TEX_RGBA32F)
        t += 1
    xf = g[f"{tag}_inst_xf"]
    for i, (mesh, mat) in enumerate(zip(g[f"{tag}_inst_mesh"], g[f"{tag}_inst_mat"])):
        rows = [xf[i, k].reshape(4, 4).T for k in range(3)]  # column-major storage -> row-major
        sb.add_instance(int(mesh), int(mat), rows[0], inverse=rows[1], inv_transpose=rows[2])
    sb.camera = CameraDesc.from_buffer_copy(g[f"{tag}_camera"].tobytes())
    sb.trace_depth = int(g[f"{tag}_trace_depth"][0])
    if f"{tag}_env" in g:
        sb.set_env(g[f"{tag}_env"])
    return sb
