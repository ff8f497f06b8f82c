"""Field-by-field comparison of two scene descriptions (lux_scene_desc) -- test helper for the
glTF loader parity (luxion_b200/gltf.py against the reference's Scene::loadFromGLTF)."""
import numpy as np

MAT_FIELDS = ("albedo_tex", "alpha", "alpha_mode", "alpha_cutoff", "emission_strength", "emissive_tex", "roughness",
              "metallic", "normal_tex", "metallic_roughness_tex", "transmission", "ior")
TT = ("albedo_tt", "emissive_tt", "normal_tt", "metallic_roughness_tt")


def mesh_arrays(d, i):
    m = d.meshes[d.instances[i].mesh]
    out = {"positions": np.ctypeslib.as_array(m.positions, shape=(m.num_verts * 3,)).copy(),
           "indices": np.ctypeslib.as_array(m.indices, shape=(m.num_tris * 3,)).copy()}
    if m.normals:
        out["normals"] = np.ctypeslib.as_array(m.normals, shape=(m.num_verts * 3,)).copy()
    if m.uvs:
        out["uvs"] = np.ctypeslib.as_array(m.uvs, shape=(m.num_verts * 2,)).copy()
    return out


def texels(d, t):
    """Texture t as float32 RGBA in [0, 1] (unorm formats converted as c / 255, c / 65535)."""
    x = d.textures[t]
    n = x.width * x.height * 4
    import ctypes
    if x.format == 0:
        a = np.ctypeslib.as_array(ctypes.cast(x.data, ctypes.POINTER(ctypes.c_uint8)), shape=(n,))
        return a.astype(np.float32) / np.float32(255.0)
    if x.format == 1:
        a = np.ctypeslib.as_array(ctypes.cast(x.data, ctypes.POINTER(ctypes.c_uint16)), shape=(n,))
        return a.astype(np.float32) / np.float32(65535.0)
    return np.ctypeslib.as_array(ctypes.cast(x.data, ctypes.POINTER(ctypes.c_float)), shape=(n,)).copy()


def compare_descs(a, b):
    """List of differences between scene descriptions a and b (empty when they agree)."""
    diffs = []
    for k in ("num_instances", "num_materials", "num_textures", "trace_depth", "env_width", "env_height"):
        if getattr(a, k) != getattr(b, k):
            diffs.append((k, getattr(a, k), getattr(b, k)))
    if diffs:
        return diffs
    ca, cb = a.camera, b.camera
    for k in ("width", "height"):
        if getattr(ca, k) != getattr(cb, k):
            diffs.append(("camera." + k, getattr(ca, k), getattr(cb, k)))
    for k in ("position", "look_at", "view", "up", "right", "fov", "pixel_length"):
        if not np.array_equal(np.array(getattr(ca, k)), np.array(getattr(cb, k))):
            diffs.append(("camera." + k, list(getattr(ca, k)), list(getattr(cb, k))))
    for i in range(a.num_instances):
        ia, ib = a.instances[i], b.instances[i]
        if ia.material != ib.material:
            diffs.append((f"instance {i} material", ia.material, ib.material))
        for k in ("transform", "inverse", "inv_transpose"):
            if not np.array_equal(np.array(getattr(ia, k)), np.array(getattr(ib, k))):
                diffs.append((f"instance {i} {k}", list(getattr(ia, k)), list(getattr(ib, k))))
        ma, mb = mesh_arrays(a, i), mesh_arrays(b, i)
        if set(ma) != set(mb):
            diffs.append((f"instance {i} mesh attributes", sorted(ma), sorted(mb)))
            continue
        for k in ma:
            if ma[k].shape != mb[k].shape or not np.array_equal(ma[k], mb[k]):
                diffs.append((f"instance {i} {k}", ma[k].shape, mb[k].shape))
    for k in range(a.num_materials):
        x, y = a.materials[k], b.materials[k]
        if not np.array_equal(np.array(x.color), np.array(y.color)):
            diffs.append((f"material {k} color", list(x.color), list(y.color)))
        if not np.array_equal(np.array(x.emission_color), np.array(y.emission_color)):
            diffs.append((f"material {k} emission_color", list(x.emission_color), list(y.emission_color)))
        for f in MAT_FIELDS:
            if getattr(x, f) != getattr(y, f):
                diffs.append((f"material {k} {f}", getattr(x, f), getattr(y, f)))
        for f in TT:
            p, q = getattr(x, f), getattr(y, f)
            if list(p.offset) != list(q.offset) or list(p.scale) != list(q.scale) or p.rotation != q.rotation:
                diffs.append((f"material {k} {f}",))
    for t in range(a.num_textures):
        if (a.textures[t].width, a.textures[t].height) != (b.textures[t].width, b.textures[t].height):
            diffs.append((f"texture {t} size",))
        elif not np.array_equal(texels(a, t), texels(b, t)):
            diffs.append((f"texture {t} texels",))
    if a.env_data and b.env_data:
        import ctypes
        n = a.env_width * a.env_height * 4
        ea = np.ctypeslib.as_array(ctypes.cast(a.env_data, ctypes.POINTER(ctypes.c_float)), shape=(n,))
        eb = np.ctypeslib.as_array(ctypes.cast(b.env_data, ctypes.POINTER(ctypes.c_float)), shape=(n,))
        if not np.array_equal(ea, eb):
            diffs.append(("environment texels", float(np.abs(ea - eb).max())))
    return diffs
