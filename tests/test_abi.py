"""C-ABI checks that need no GPU: the library loads, exports every entry point the header
declares, its structures have the header's layout, arguments are validated before any device
work, and the procedural scenes are generated on the host."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import luxion_b200 as lx
from luxion_b200 import _ffi
from luxion_b200._ffi import default_options
from conftest import cuda_device_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "luxion.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(lux_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = lx.lib()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    # the Python mirror binds every declared entry point
    assert set(names) <= set(lx.SIGNATURES), set(names) - set(lx.SIGNATURES)


STRUCTS = {
    "lux_texture_desc": _ffi.TextureDesc, "lux_tex_transform": _ffi.TexTransform,
    "lux_material_desc": _ffi.MaterialDesc, "lux_mesh_desc": _ffi.MeshDesc,
    "lux_instance_desc": _ffi.InstanceDesc, "lux_camera_desc": _ffi.CameraDesc,
    "lux_scene_desc": _ffi.SceneDesc, "lux_options": _ffi.Options, "lux_stats": _ffi.Stats,
    "lux_random_scene_params": _ffi.RandomSceneParams, "lux_job_desc": _ffi.JobDesc,
    "lux_engine_config": _ffi.EngineConfig, "lux_job_status": _ffi.JobStatus,
    "lux_engine_stats": _ffi.EngineStats, "lux_scene_stats": _ffi.SceneStats,
}


def test_struct_layouts_match_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            a, b, c = ln.split()
            got[(a, b)] = int(c)
    for cname, py in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_default_options_match_reference_defaults():
    o = _ffi.Options()
    lx.lib().lux_default_options(C.byref(o))
    # PathTracerOptions (include/pathtrace/pathtracer_options.h:3-11): ACES, intensity 1, NEE off
    assert o.color_mode == _ffi.TONEMAP_ACES and o.envmap_intensity == 1.0
    assert o.direct_light_sampling == 0 and o.env_importance_sampling == 0
    p = default_options()
    assert (p.color_mode, p.envmap_intensity, p.use_graph) == (o.color_mode, o.envmap_intensity, o.use_graph)


def test_init_validates_before_touching_a_device():
    L = lx.lib()
    h = C.c_void_p()
    assert L.lux_init(None, None, C.byref(h)) == -1
    assert L.lux_init(None, None, None) == -1
    # a mesh index outside the vertex range is rejected
    from luxion_b200.scene_builder import SceneBuilder
    sb = SceneBuilder(8, 8)
    m = sb.add_mesh([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 5]])
    sb.add_instance(m, sb.add_material())
    assert L.lux_init(sb.desc_ptr, None, C.byref(h)) == -1
    assert b"index out of range" in L.lux_last_error()
    # -dmis without emitters is rejected like src/main.cpp:155-160 (needs a device to reach)
    assert L.lux_free(None) == 0


@pytest.mark.skipif(cuda_device_available(), reason="a GPU is present")
def test_init_without_device_reports_no_device():
    s = lx.cornell36(16, 16)
    with pytest.raises(lx.LuxError) as e:
        lx.Renderer(s)
    assert e.value.code == -3


def test_reference_shaped_interface_errors_before_init():
    lx.pathtraceFree()
    with pytest.raises(lx.LuxError) as e:
        lx.pathtrace(0, 0, 1)
    assert e.value.code == -7
    with pytest.raises(lx.LuxError):
        lx.copyImageToHost()


def test_procedural_scenes():
    c = lx.cornell36(256, 256)
    assert c.instanced_tris == 36 and c.width == 256 and c.desc.trace_depth == 8
    d = c.desc
    emissive = [i for i in range(d.num_instances)
                if max(d.materials[d.instances[i].material].emission_color) > 0]
    assert len(emissive) == 1
    r = lx.random_scene(num_instances=20, total_tris=60000, min_tris=2000, max_tris=5000, num_emissive=3,
                        num_textures=2, texture_size=32, env_width=64, env_height=32, width=32, height=32)
    assert abs(r.instanced_tris - 60000) < 6000
    assert r.desc.num_instances == 20 and r.desc.env_width == 64
    # seeded: the same parameters give the same scene
    r2 = lx.random_scene(num_instances=20, total_tris=60000, min_tris=2000, max_tris=5000, num_emissive=3,
                         num_textures=2, texture_size=32, env_width=64, env_height=32, width=32, height=32)
    m1, m2 = r.desc.meshes[3], r2.desc.meshes[3]
    a = np.ctypeslib.as_array(m1.positions, shape=(m1.num_verts * 3,))
    b = np.ctypeslib.as_array(m2.positions, shape=(m2.num_verts * 3,))
    assert np.array_equal(a, b)
    f = lx.furnace(16, 16, 4)
    assert f.desc.env_data is not None and f.desc.num_instances == 1


def test_static_trace_limit_matches_header():
    text = open(HEADER).read()
    m = re.search(r"#define LUX_TRACE_STATIC_MAX_RAYS (\d+)", text)
    assert m and int(m.group(1)) == _ffi.TRACE_STATIC_MAX_RAYS


def test_debug_views_validated_before_touching_a_device():
    from luxion_b200._ffi import default_options
    L = lx.lib()
    s = lx.cornell36(8, 8)
    h = C.c_void_p()
    for kw, msg in ((dict(material_debug_mode=7), b"material_debug_mode"), (dict(material_debug_mode=-1), b"0..6"),
                    (dict(debug_bvh=3), b"debug_bvh"), (dict(material_debug_mode=2, debug_bvh=1), b"exclusive")):
        o = default_options(**kw)
        assert L.lux_init(s.desc_ptr, C.byref(o), C.byref(h)) != 0
        assert msg in L.lux_last_error()
    # the job engine renders the production path only
    o = default_options(debug_bvh=1)
    scenes = (C.POINTER(_ffi.SceneDesc) * 1)(s.desc_ptr)
    e = C.c_void_p()
    assert L.lux_engine_create(scenes, 1, C.byref(o), None, C.byref(e)) == -5
    assert b"debug views" in L.lux_last_error()
