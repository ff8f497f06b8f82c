"""Build a lux_scene_desc from numpy arrays (a caller-made scene, the analogue of the
reference's glTF-loaded Scene, include/scene.h:10-48).

The builder keeps every array alive for as long as it exists; the descriptor it returns
points into those arrays.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional

import numpy as np

from . import _ffi
from ._ffi import CameraDesc, InstanceDesc, MaterialDesc, MeshDesc, SceneDesc, TextureDesc


def default_material(**kw) -> MaterialDesc:
    m = MaterialDesc()
    m.color[:] = (1.0, 1.0, 1.0)
    m.albedo_tex = -1
    m.alpha = 1.0
    m.alpha_mode = _ffi.ALPHA_OPAQUE
    m.alpha_cutoff = 0.5
    m.emission_strength = 1.0
    m.emission_color[:] = (0.0, 0.0, 0.0)
    m.emissive_tex = -1
    m.roughness = 1.0
    m.metallic = 0.0
    m.normal_tex = -1
    m.metallic_roughness_tex = -1
    m.transmission = 0.0
    m.ior = 1.55
    for tt in (m.albedo_tt, m.emissive_tt, m.normal_tt, m.metallic_roughness_tt):
        tt.offset[:] = (0.0, 0.0)
        tt.scale[:] = (1.0, 1.0)
        tt.rotation = 0.0
    for k, v in kw.items():
        if k in ("color", "emission_color"):
            getattr(m, k)[:] = v
        else:
            setattr(m, k, v)
    return m


def look_at_camera(width: int, height: int, pos, look, fovy_deg: float = 45.0) -> CameraDesc:
    """Camera with the conventions of the reference's glTF loader
    (src/scene/scene_load_gltf.cpp:465-500)."""
    pos = np.asarray(pos, np.float64)
    look = np.asarray(look, np.float64)
    v = look - pos
    v /= np.linalg.norm(v)
    r = np.cross(v, [0.0, 1.0, 0.0])
    r /= np.linalg.norm(r)
    u = np.cross(r, v)
    c = CameraDesc()
    c.width, c.height = width, height
    c.position[:] = pos.astype(np.float32)
    c.look_at[:] = (pos + v).astype(np.float32)
    c.view[:] = v.astype(np.float32)
    c.right[:] = r.astype(np.float32)
    c.up[:] = u.astype(np.float32)
    yscaled = np.float32(np.tan(np.float32(0.5) * np.float32(fovy_deg) * np.float32(np.pi / 180)))
    xscaled = np.float32(yscaled * np.float32(width) / np.float32(height))
    c.fov[:] = (float(2 * np.arctan(xscaled) * 180 / np.pi), fovy_deg)
    c.pixel_length[:] = (float(2 * xscaled / np.float32(width)), float(2 * yscaled / np.float32(height)))
    return c


class SceneBuilder:
    def __init__(self, width: int = 64, height: int = 64, trace_depth: int = 8):
        self._keep: List[object] = []
        self.meshes: List[MeshDesc] = []
        self.instances: List[InstanceDesc] = []
        self.materials: List[MaterialDesc] = []
        self.textures: List[TextureDesc] = []
        self.camera = look_at_camera(width, height, (0, 0, 3), (0, 0, 0))
        self.trace_depth = trace_depth
        self.env = None
        self._desc: Optional[SceneDesc] = None

    def _hold(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a)
        self._keep.append(a)
        return a

    def add_mesh(self, positions, indices, normals=None, uvs=None) -> int:
        p = self._hold(np.asarray(positions, np.float32).reshape(-1, 3))
        i = self._hold(np.asarray(indices, np.uint32).reshape(-1, 3))
        m = MeshDesc()
        m.num_verts = p.shape[0]
        m.num_tris = i.shape[0]
        m.positions = p.ctypes.data_as(C.POINTER(C.c_float))
        m.indices = i.ctypes.data_as(C.POINTER(C.c_uint32))
        m.normals = None
        m.uvs = None
        if normals is not None:
            n = self._hold(np.asarray(normals, np.float32).reshape(-1, 3))
            m.normals = n.ctypes.data_as(C.POINTER(C.c_float))
        if uvs is not None:
            u = self._hold(np.asarray(uvs, np.float32).reshape(-1, 2))
            m.uvs = u.ctypes.data_as(C.POINTER(C.c_float))
        self.meshes.append(m)
        return len(self.meshes) - 1

    def add_material(self, mat: Optional[MaterialDesc] = None, **kw) -> int:
        self.materials.append(mat if mat is not None else default_material(**kw))
        return len(self.materials) - 1

    def add_texture(self, texels: np.ndarray, fmt: int) -> int:
        h, w = texels.shape[:2]
        dt = {_ffi.TEX_RGBA8: np.uint8, _ffi.TEX_RGBA16: np.uint16, _ffi.TEX_RGBA32F: np.float32,
              _ffi.TEX_RGBA16F: np.float16}[fmt]
        a = self._hold(np.asarray(texels, dt).reshape(h, w, 4))
        t = TextureDesc()
        t.width, t.height, t.format = w, h, fmt
        t.data = a.ctypes.data
        self.textures.append(t)
        return len(self.textures) - 1

    def add_instance(self, mesh: int, material: int, transform=None, inverse=None, inv_transpose=None) -> int:
        """Place a mesh. Matrices are row-major 4x4; the inverse and inverse transpose are
        derived in double unless given."""
        M = np.eye(4, dtype=np.float64) if transform is None else np.asarray(transform, np.float64)
        inv = np.linalg.inv(M) if inverse is None else np.asarray(inverse, np.float64)
        inv_t = inv.T if inv_transpose is None else np.asarray(inv_transpose, np.float64)
        d = InstanceDesc()
        d.mesh, d.material, d.has_inverse = mesh, material, 1
        # column-major (glm) storage
        d.transform[:] = M.T.reshape(-1).astype(np.float32)
        d.inverse[:] = inv.T.reshape(-1).astype(np.float32)
        d.inv_transpose[:] = inv_t.T.reshape(-1).astype(np.float32)
        self.instances.append(d)
        return len(self.instances) - 1

    def set_env(self, texels: np.ndarray, half: bool = False):
        h, w = texels.shape[:2]
        a = self._hold(np.asarray(texels, np.float16 if half else np.float32).reshape(h, w, 4))
        self.env = (w, h, _ffi.TEX_RGBA16F if half else _ffi.TEX_RGBA32F, a)

    def build(self) -> SceneDesc:
        d = SceneDesc()
        ma = (MeshDesc * len(self.meshes))(*self.meshes)
        ia = (InstanceDesc * len(self.instances))(*self.instances)
        mt = (MaterialDesc * len(self.materials))(*self.materials)
        ta = (TextureDesc * max(1, len(self.textures)))(*self.textures)
        self._keep += [ma, ia, mt, ta]
        d.num_meshes, d.num_instances = len(self.meshes), len(self.instances)
        d.num_materials, d.num_textures = len(self.materials), len(self.textures)
        d.meshes = C.cast(ma, C.POINTER(MeshDesc))
        d.instances = C.cast(ia, C.POINTER(InstanceDesc))
        d.materials = C.cast(mt, C.POINTER(MaterialDesc))
        d.textures = C.cast(ta, C.POINTER(TextureDesc)) if self.textures else None
        d.camera = self.camera
        d.trace_depth = self.trace_depth
        if self.env is not None:
            d.env_width, d.env_height, d.env_format = self.env[0], self.env[1], self.env[2]
            d.env_data = self.env[3].ctypes.data
        else:
            d.env_data = None
        self._desc = d
        return d

    # the HostScene protocol used by Renderer and the oracle bindings
    @property
    def desc_ptr(self):
        if self._desc is None:
            self.build()
        return C.pointer(self._desc)

    @property
    def desc(self) -> SceneDesc:
        if self._desc is None:
            self.build()
        return self._desc

    @property
    def width(self) -> int:
        return self.camera.width

    @property
    def height(self) -> int:
        return self.camera.height
