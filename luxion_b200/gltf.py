"""glTF 2.0 scenes (.glb, or .gltf with embedded or external buffers) into a SceneBuilder,
following the reference's loader (src/scene/scene_load_gltf.cpp:61-529):

- material 0 is the reference's default material, red microfacet (:85-89); glTF material k
  becomes material k + 1;
- base colour and alpha from baseColorFactor, metallic and roughness factors (glTF defaults
  1), emission = emissiveFactor with KHR_materials_emissive_strength (default 1), IOR from
  KHR_materials_ior (default 1.55), KHR_materials_transmission, alphaMode and alphaCutoff,
  the base colour, emissive, normal and metallic-roughness textures with their
  KHR_texture_transform (:150-240);
- every triangle primitive of every node becomes one instance with the node's global
  transform (matrix, or translation * rotation * scale, composed down the hierarchy), its
  positions, normalised normals, first UV set and indices (:242-420);
- the camera node gives the pinhole camera: the short side of the resolution is 1000 pixels
  and the other follows the aspect ratio, the view is -z of the node, and the trace depth
  is 8 (:429-488).
Images are decoded with Pillow to RGBA (8 or 16 bits per channel).
"""
from __future__ import annotations

import base64
import io
import json
import math
import os
import struct
from typing import List, Optional

import numpy as np

from . import _ffi, glmf
from .scene_builder import SceneBuilder, default_material

_COMPONENT = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


class GltfError(ValueError):
    pass


def _read(path: str):
    with open(path, "rb") as f:
        data = f.read()
    base = os.path.dirname(os.path.abspath(path))
    if data[:4] == b"glTF":
        _, version, length = struct.unpack("<4sII", data[:12])
        if version != 2:
            raise GltfError(f"glTF version {version} is not supported")
        pos, doc, binchunk = 12, None, b""
        while pos < min(length, len(data)):
            clen, ctype = struct.unpack("<II", data[pos:pos + 8])
            chunk = data[pos + 8:pos + 8 + clen]
            if ctype == 0x4E4F534A:
                doc = json.loads(chunk.decode("utf-8"))
            elif ctype == 0x004E4942:
                binchunk = chunk
            pos += 8 + clen
        if doc is None:
            raise GltfError("no JSON chunk")
    else:
        doc, binchunk = json.loads(data.decode("utf-8")), b""
    buffers = []
    for i, b in enumerate(doc.get("buffers", [])):
        uri = b.get("uri")
        if uri is None:
            buffers.append(binchunk)
        elif uri.startswith("data:"):
            buffers.append(base64.b64decode(uri.split(",", 1)[1]))
        else:
            with open(os.path.join(base, uri), "rb") as f:
                buffers.append(f.read())
    return doc, buffers, base


class _Model:
    def __init__(self, doc, buffers, base):
        self.doc, self.buffers, self.base = doc, buffers, base

    def view_bytes(self, vi: int) -> bytes:
        v = self.doc["bufferViews"][vi]
        b = self.buffers[v["buffer"]]
        off = v.get("byteOffset", 0)
        return b[off:off + v["byteLength"]]

    def accessor(self, ai: int) -> np.ndarray:
        a = self.doc["accessors"][ai]
        dt = np.dtype(_COMPONENT[a["componentType"]])
        nc = _NCOMP[a["type"]]
        count = a["count"]
        if "bufferView" not in a:
            return np.zeros((count, nc), dt)
        v = self.doc["bufferViews"][a["bufferView"]]
        raw = self.view_bytes(a["bufferView"])
        off = a.get("byteOffset", 0)
        stride = v.get("byteStride", 0) or dt.itemsize * nc
        out = np.empty((count, nc), dt)
        if stride == dt.itemsize * nc:
            out[:] = np.frombuffer(raw, dt, count * nc, off).reshape(count, nc)
        else:
            for i in range(count):
                out[i] = np.frombuffer(raw, dt, nc, off + i * stride)
        return out

    def image(self, ii: int) -> np.ndarray:
        from PIL import Image
        im = self.doc["images"][ii]
        if "bufferView" in im:
            data = self.view_bytes(im["bufferView"])
        elif im.get("uri", "").startswith("data:"):
            data = base64.b64decode(im["uri"].split(",", 1)[1])
        else:
            with open(os.path.join(self.base, im["uri"]), "rb") as f:
                data = f.read()
        img = Image.open(io.BytesIO(data))
        if img.mode in ("I;16", "I;16B", "I;16L") or img.mode.startswith("RGBA;16") or img.mode == "I":
            arr = np.asarray(img).astype(np.uint16)
            if arr.ndim == 2:
                arr = np.stack([arr, arr, arr, np.full_like(arr, 65535)], axis=2)
            return arr
        return np.asarray(img.convert("RGBA"), np.uint8)


def _libm():
    import ctypes
    import ctypes.util
    lm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    for fn in (lm.tanf, lm.atanf):
        fn.restype, fn.argtypes = ctypes.c_float, [ctypes.c_float]
    return lm


def _node_matrix(node) -> np.ndarray:
    """The node's local matrix as the reference composes it in float (glm column-major):
    the matrix if given, else translate(I, t) * mat4_cast(q) then scale(., s)
    (src/scene/scene_load_gltf.cpp:250-290)."""
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).reshape(4, 4).astype(np.float32)  # columns in the file
    M = glmf.identity()
    if "translation" in node:
        M = glmf.translate(M, node["translation"])
    if "rotation" in node:
        x, y, z, w = node["rotation"]
        M = glmf.mul(M, glmf.mat4_cast(w, x, y, z))
    if "scale" in node:
        M = glmf.scale(M, node["scale"])
    return M


def _normalize_f32(v: np.ndarray) -> np.ndarray:
    """glm::normalize in float: v * (1 / sqrt(dot(v, v))), dot = (x*x + y*y) + z*z."""
    v = v.astype(np.float32)
    d = (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]
    inv = np.float32(1.0) / np.sqrt(d)
    return v * inv[:, None]


def _tex_transform(info: Optional[dict], tt) -> None:
    ext = (info or {}).get("extensions", {}).get("KHR_texture_transform")
    if not ext:
        return
    if "offset" in ext:
        tt.offset[:] = [float(x) for x in ext["offset"]]
    if "scale" in ext:
        tt.scale[:] = [float(x) for x in ext["scale"]]
    if "rotation" in ext:
        tt.rotation = float(ext["rotation"])


def load(path: str) -> SceneBuilder:
    """The scene of a glTF file as a SceneBuilder (camera, trace depth 8, no environment map)."""
    doc, buffers, base = _read(path)
    M = _Model(doc, buffers, base)
    sb = SceneBuilder()
    sb.trace_depth = 8
    # textures: glTF texture index k -> texture k
    for t in doc.get("textures", []):
        arr = M.image(t["source"])
        sb.add_texture(arr, _ffi.TEX_RGBA16 if arr.dtype == np.uint16 else _ffi.TEX_RGBA8)
    ntex = len(doc.get("textures", []))

    def tex_index(info):
        if not info or "index" not in info:
            return -1
        if not 0 <= info["index"] < ntex:
            raise GltfError(f"texture index {info['index']} out of range")
        return int(info["index"])

    # materials: 0 = the reference's default (red), then the file's
    red = default_material(color=(1.0, 0.0, 0.0), roughness=0.0, metallic=0.0, ior=0.0, emission_strength=0.0)
    sb.add_material(red)
    for m in doc.get("materials", []):
        pbr = m.get("pbrMetallicRoughness", {})
        base_color = pbr.get("baseColorFactor", [1.0, 1.0, 1.0, 1.0])
        ext = m.get("extensions", {})
        mat = default_material()
        mat.color[:] = [float(x) for x in base_color[:3]]
        mat.alpha = float(base_color[3]) if len(base_color) > 3 else 1.0
        mat.metallic = float(pbr.get("metallicFactor", 1.0))
        mat.roughness = float(pbr.get("roughnessFactor", 1.0))
        mat.emission_strength = float(ext.get("KHR_materials_emissive_strength", {}).get("emissiveStrength", 1.0))
        mat.emission_color[:] = [float(x) for x in m.get("emissiveFactor", [0.0, 0.0, 0.0])]
        mat.ior = float(ext.get("KHR_materials_ior", {}).get("ior", 1.55))
        mat.transmission = float(ext.get("KHR_materials_transmission", {}).get("transmissionFactor", 0.0))
        mode = m.get("alphaMode", "OPAQUE")
        mat.alpha_mode = {"MASK": _ffi.ALPHA_MASK, "BLEND": _ffi.ALPHA_BLEND}.get(mode, _ffi.ALPHA_OPAQUE)
        mat.alpha_cutoff = float(m.get("alphaCutoff", 0.5))
        mat.albedo_tex = tex_index(pbr.get("baseColorTexture"))
        mat.metallic_roughness_tex = tex_index(pbr.get("metallicRoughnessTexture"))
        mat.emissive_tex = tex_index(m.get("emissiveTexture"))
        mat.normal_tex = tex_index(m.get("normalTexture"))
        _tex_transform(pbr.get("baseColorTexture"), mat.albedo_tt)
        _tex_transform(pbr.get("metallicRoughnessTexture"), mat.metallic_roughness_tt)
        _tex_transform(m.get("emissiveTexture"), mat.emissive_tt)
        _tex_transform(m.get("normalTexture"), mat.normal_tt)
        sb.add_material(mat)

    mesh_cache = {}

    def prim_mesh(mi: int, pi: int):
        key = (mi, pi)
        if key in mesh_cache:
            return mesh_cache[key]
        prim = doc["meshes"][mi]["primitives"][pi]
        attrs = prim.get("attributes", {})
        if prim.get("mode", 4) != 4 or "POSITION" not in attrs:
            mesh_cache[key] = None
            return None
        pos = M.accessor(attrs["POSITION"]).astype(np.float32)
        nrm = _normalize_f32(M.accessor(attrs["NORMAL"])) if "NORMAL" in attrs else None
        uv = M.accessor(attrs["TEXCOORD_0"]).astype(np.float32) if "TEXCOORD_0" in attrs else None
        if "indices" in prim:
            idx = M.accessor(prim["indices"]).reshape(-1).astype(np.uint32)
        else:
            idx = np.arange(pos.shape[0], dtype=np.uint32)
        if idx.size % 3 or idx.size == 0:
            raise GltfError(f"mesh {mi} primitive {pi}: index count {idx.size} is not a positive multiple of 3")
        mesh_cache[key] = (sb.add_mesh(pos, idx.reshape(-1, 3), normals=nrm, uvs=uv),
                           prim.get("material", -1))
        return mesh_cache[key]

    camera = []
    nodes = doc.get("nodes", [])

    def visit(ni: int, parent: np.ndarray):
        node = nodes[ni]
        G = glmf.mul(parent, _node_matrix(node))  # global = parent * local, in float
        if "mesh" in node:
            inv, inv_t = glmf.inverse(G), glmf.inverse_transpose(G)
            for pi in range(len(doc["meshes"][node["mesh"]]["primitives"])):
                pm = prim_mesh(node["mesh"], pi)
                if pm is None:
                    continue
                mesh, mat = pm
                # row-major for the builder; inverse and inverse transpose as glm computes them
                sb.add_instance(mesh, mat + 1 if mat >= 0 else 0, G.T, inverse=inv.T, inv_transpose=inv_t.T)
        if "camera" in node:
            if camera:
                raise GltfError("more than one camera in the scene")
            camera.append((node["camera"], G))
        for c in node.get("children", []):
            visit(c, G)

    scenes = doc.get("scenes", [])
    si = doc.get("scene", 0)
    roots = scenes[si]["nodes"] if scenes else list(range(len(nodes)))
    for r in roots:
        visit(r, glmf.identity())
    if not sb.instances:
        raise GltfError("no triangle meshes in the scene")
    if not camera:
        raise GltfError("no camera in the scene")
    ci, G = camera[0]
    persp = doc["cameras"][ci].get("perspective", {})
    aspect = float(persp.get("aspectRatio", 1.0))
    if aspect >= 1.0:
        h = 1000
        w = int(np.float32(aspect) * np.float32(h))
    else:
        w = 1000
        h = int(np.float32(w) / np.float32(aspect))
    # glm::degrees of the double yfov, stored as float
    fovy = float(np.float32(persp.get("yfov", math.radians(45.0)) * 57.295779513082320876798154814105))
    cam = _ffi.CameraDesc()
    cam.width, cam.height = w, h
    eye = G[3][:3]
    view = -glmf.normalize(G[2][:3])
    right = glmf.normalize(G[0][:3])
    up = glmf.normalize(G[1][:3])
    cam.position[:] = [float(x) for x in eye]
    cam.view[:] = [float(x) for x in view]
    cam.right[:] = [float(x) for x in right]
    cam.up[:] = [float(x) for x in up]
    cam.look_at[:] = [float(x) for x in (eye + view)]
    pi = np.float32(3.1415926535897932384626422832795028841971)
    # float tan / atan of the C math library (the float overloads the loader calls), float
    # arithmetic around them (scene_load_gltf.cpp:485-491)
    yscaled = np.float32(_libm().tanf(float(np.float32(0.5) * np.float32(fovy) * (pi / np.float32(180)))))
    xscaled = (yscaled * np.float32(w)) / np.float32(h)
    fovx = (np.float32(2) * np.float32(_libm().atanf(float(xscaled))) * np.float32(180)) / pi
    cam.fov[:] = [float(fovx), fovy]
    cam.pixel_length[:] = [float(np.float32(2) * xscaled / np.float32(w)), float(np.float32(2) * yscaled / np.float32(h))]
    sb.camera = cam
    return sb


def save_glb(path: str, meshes: List[dict], materials: List[dict], nodes: List[dict], camera: dict,
             images: Optional[List[np.ndarray]] = None) -> None:
    """A minimal .glb writer (float positions / normals / uvs, u32 indices, PNG images): the
    format the tests load back, so that no outside asset is needed."""
    from PIL import Image
    blob = bytearray()
    views, accessors = [], []

    def add_view(data: bytes) -> int:
        while len(blob) % 4:
            blob.append(0)
        views.append({"buffer": 0, "byteOffset": len(blob), "byteLength": len(data)})
        blob.extend(data)
        return len(views) - 1

    def add_accessor(arr: np.ndarray, ctype: int, typ: str) -> int:
        accessors.append({"bufferView": add_view(arr.tobytes()), "componentType": ctype, "count": int(arr.shape[0]),
                          "type": typ})
        return len(accessors) - 1

    gl_meshes = []
    for m in meshes:
        attrs = {"POSITION": add_accessor(np.asarray(m["positions"], np.float32), 5126, "VEC3")}
        if m.get("normals") is not None:
            attrs["NORMAL"] = add_accessor(np.asarray(m["normals"], np.float32), 5126, "VEC3")
        if m.get("uvs") is not None:
            attrs["TEXCOORD_0"] = add_accessor(np.asarray(m["uvs"], np.float32), 5126, "VEC2")
        prim = {"attributes": attrs, "mode": 4,
                "indices": add_accessor(np.asarray(m["indices"], np.uint32).reshape(-1, 1), 5125, "SCALAR")}
        if m.get("material") is not None:
            prim["material"] = m["material"]
        gl_meshes.append({"primitives": [prim]})
    gl_images, gl_textures = [], []
    for img in images or []:
        buf = io.BytesIO()
        Image.fromarray(np.asarray(img, np.uint8), "RGBA").save(buf, format="PNG")
        gl_images.append({"bufferView": add_view(buf.getvalue()), "mimeType": "image/png"})
        gl_textures.append({"source": len(gl_images) - 1})
    children = {c for n in nodes for c in n.get("children", [])}
    roots = [i for i in range(len(nodes)) if i not in children]
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": roots}],
           "nodes": nodes, "meshes": gl_meshes, "materials": materials, "accessors": accessors,
           "bufferViews": views, "buffers": [{"byteLength": len(blob)}],
           "cameras": [{"type": "perspective", "perspective": camera}]}
    if gl_images:
        doc["images"], doc["textures"] = gl_images, gl_textures
    js = json.dumps(doc).encode("utf-8")
    js += b" " * ((4 - len(js) % 4) % 4)
    while len(blob) % 4:
        blob.append(0)
    total = 12 + 8 + len(js) + 8 + len(blob)
    with open(path, "wb") as f:
        f.write(struct.pack("<4sII", b"glTF", 2, total))
        f.write(struct.pack("<II", len(js), 0x4E4F534A) + js)
        f.write(struct.pack("<II", len(blob), 0x004E4942) + bytes(blob))
