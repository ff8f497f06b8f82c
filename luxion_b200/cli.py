"""Headless command line of the renderer, with the reference's flags (src/main.cpp:81-147):

    python -m luxion_b200 SCENE [-e|--envmap ENVMAP] [-i|--iterations N] [-o|--output NAME]
                                [-dmis] [-emis] [-lock] [-debug-material N] [-debug-bvh]

SCENE is a glTF 2.0 file (.glb or .gltf, loaded as the reference's loader does: luxion_b200.gltf)
or a procedural scene: cornell (the 36-triangle Cornell box), random[:SEED[:TRIS]] (the
instanced test scene) or furnace. ENVMAP is an OpenEXR (.exr) or Radiance (.hdr) image, or a
float32 .npy array of HxWx3 or HxWx4 texels, replacing the scene's environment map. -lock is
accepted and ignored (it locks the interactive camera).
-debug-material N (1 albedo, 2 world normal, 3 normal map, 4 roughness, 5 metallic, 6 alpha) and
-debug-bvh select the debug views the reference offers in its ImGui panel
(src/app/render_imgui.cpp:336-345): PathTracerOptions::material_debug_mode and debug_bvh.
The image is written as NAME.png the way the reference's saveImage does
(src/app/save_image.cpp:42-84): the accumulated sum divided by the sample count, ACES, gamma
0.45, x mirrored, each channel clamped to [0, 1] and truncated from value * 255. A material
debug view is written as the reference displays it (src/kernels/image_kernels.cu:20-33): the
mean without tone map or gamma, x mirrored like every saved image.
"""
from __future__ import annotations

import os
import struct
import sys
import time
import zlib
from typing import List, Optional

import numpy as np

USAGE = ("Usage: %s SCENEFILE [-e|--envmap ENVMAP] [-i|--iterations N] [-o|--output NAME] [-dmis] [-emis] [-lock]\n"
         "       [-debug-material N] [-debug-bvh]\n"
         "  SCENEFILE: a .glb/.gltf file, or cornell | random[:SEED[:TRIS]] | furnace\n"
         "  -debug-material N: 1 albedo, 2 world normal, 3 normal map, 4 roughness, 5 metallic, 6 alpha")


def parse_args(argv: List[str]) -> dict:
    """Parse the reference's flags; raise ValueError with its messages on bad input."""
    out = {"scene": None, "envmap": None, "iterations": 5000, "output": None, "dmis": False, "emis": False,
           "lock": False, "debug_material": 0, "debug_bvh": False}
    i = 0
    while i < len(argv):
        a = argv[i]
        if a in ("-e", "--envmap"):
            if i + 1 >= len(argv):
                raise ValueError(f"Error: {a} requires a path")
            out["envmap"] = argv[i + 1]
            i += 1
        elif a in ("-i", "--iterations"):
            if i + 1 >= len(argv):
                raise ValueError(f"Error: {a} requires a number")
            v = argv[i + 1]
            if not v.isdigit() or int(v) <= 0:
                raise ValueError(f"Error: invalid iteration count '{v}'")
            out["iterations"] = int(v)
            i += 1
        elif a in ("-o", "--output"):
            if i + 1 >= len(argv):
                raise ValueError(f"Error: {a} requires a name")
            out["output"] = argv[i + 1]
            i += 1
        elif a == "-dmis":
            out["dmis"] = True
        elif a == "-emis":
            out["emis"] = True
        elif a == "-lock":
            out["lock"] = True
        elif a == "-debug-material":
            if i + 1 >= len(argv):
                raise ValueError(f"Error: {a} requires a number")
            v = argv[i + 1]
            if v not in ("1", "2", "3", "4", "5", "6"):
                raise ValueError(f"Error: invalid material debug mode '{v}' (1..6)")
            out["debug_material"] = int(v)
            i += 1
        elif a == "-debug-bvh":
            out["debug_bvh"] = True
        elif out["scene"] is None:
            out["scene"] = a
        else:
            raise ValueError(f"Error: unexpected argument '{a}'")
        i += 1
    if out["scene"] is None:
        raise ValueError("usage")
    if out["debug_material"] and out["debug_bvh"]:
        raise ValueError("Error: -debug-material and -debug-bvh are exclusive")
    return out


def aces(x: np.ndarray) -> np.ndarray:
    """ACESFilmHost (src/app/save_image.cpp:32-39) in float32."""
    a, b, c, d, e = (np.float32(v) for v in (2.51, 0.03, 2.43, 0.59, 0.14))
    return np.clip((x * (a * x + b)) / (x * (c * x + d) + e), np.float32(0), np.float32(1))


def to_png_bytes(image_sum: np.ndarray, samples: int, tonemap: bool = True) -> np.ndarray:
    """HxWx3 uint8 of saveImage: mean, ACES, gamma 0.45, x mirrored, clamp * 255 truncated.
    tonemap=False leaves out ACES and gamma (a material debug view)."""
    pix = image_sum.astype(np.float32) / np.float32(samples)
    if tonemap:
        pix = np.power(aces(pix), np.float32(0.45))
    pix = pix[:, ::-1, :]
    return (np.clip(pix, np.float32(0), np.float32(1)) * np.float32(255)).astype(np.uint8)


def write_png(path: str, rgb: np.ndarray) -> None:
    """8-bit RGB PNG, filter 0 on every row."""
    h, w, _ = rgb.shape
    raw = b"".join(b"\x00" + np.ascontiguousarray(rgb[y]).tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def read_png(path: str) -> np.ndarray:
    """Reader for the PNGs write_png makes (8-bit RGB, filter 0)."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, 3).copy()


def load_envmap(path: str) -> np.ndarray:
    """HxWx4 float32 RGBA texels of an .exr / .hdr image (alpha 1 where the file has none)
    or of an .npy array."""
    if path.lower().endswith(".npy"):
        env = np.load(path).astype(np.float32)
    else:
        os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
        import cv2
        env = cv2.imread(path, cv2.IMREAD_UNCHANGED)
        if env is None:
            raise ValueError(f"Error: cannot read environment map '{path}'")
        env = env.astype(np.float32)
        if env.ndim == 3 and env.shape[2] >= 3:   # OpenCV gives BGR(A)
            env = np.concatenate([env[..., 2::-1], env[..., 3:]], axis=2)
    if env.ndim != 3 or env.shape[2] not in (3, 4):
        raise ValueError(f"Error: environment map '{path}' must have 3 or 4 channels")
    if env.shape[2] == 3:
        env = np.concatenate([env, np.ones(env.shape[:2] + (1,), np.float32)], axis=2)
    return np.ascontiguousarray(env)


def make_scene(spec: str):
    import luxion_b200 as lx
    if spec.lower().endswith((".glb", ".gltf")):
        from luxion_b200 import gltf
        try:
            return gltf.load(spec)
        except (OSError, ValueError, KeyError) as e:
            raise ValueError(f"Error: cannot load scene '{spec}': {e}")
    parts = spec.split(":")
    name = parts[0].lower()
    if name in ("cornell", "cornell36"):
        return lx.cornell36(256, 256)
    if name == "random":
        kw = {}
        if len(parts) > 1:
            kw["seed"] = int(parts[1])
        if len(parts) > 2:
            kw["total_tris"] = int(parts[2])
        return lx.random_scene(**kw)
    if name == "furnace":
        return lx.furnace()
    raise ValueError(f"Error: cannot load scene '{spec}': give a .glb/.gltf file or one of the procedural "
                     "scenes cornell, random[:SEED[:TRIS]], furnace")


def main(argv: Optional[List[str]] = None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        a = parse_args(argv)
    except ValueError as e:
        print(USAGE % "luxion_b200" if str(e) == "usage" else e)
        return 1
    import luxion_b200 as lx
    from luxion_b200 import _ffi
    try:
        scene = make_scene(a["scene"])
    except ValueError as e:
        print(e)
        return 1
    keep = None
    if a["envmap"]:
        try:
            keep = env = load_envmap(a["envmap"])
        except (OSError, ValueError) as e:
            print(e)
            return 1
        d = scene.desc
        d.env_width, d.env_height, d.env_format = env.shape[1], env.shape[0], _ffi.TEX_RGBA32F
        d.env_data = keep.ctypes.data
    opt = lx.default_options(direct_light_sampling=int(a["dmis"]), env_importance_sampling=int(a["emis"]),
                             material_debug_mode=a["debug_material"], debug_bvh=int(a["debug_bvh"]))
    try:
        r = lx.Renderer(scene, opt)
    except lx.LuxError as e:
        print(f"Error: {e}")
        return 1
    t0 = time.perf_counter()
    r.render(1, a["iterations"])
    img = r.image_sum()
    dt = time.perf_counter() - t0
    st = r.stats()
    r.close()
    name = a["output"] or f"{a['scene'].replace(':', '_')}.{a['iterations']}samp"
    out = name + ".png"
    if os.path.dirname(out):
        os.makedirs(os.path.dirname(out), exist_ok=True)
    write_png(out, to_png_bytes(img, a["iterations"], tonemap=not a["debug_material"]))
    rays = st["rays_radiance"] + st["rays_shadow"]
    print(f"Saved {out}. {a['iterations']} samples of {img.shape[1]}x{img.shape[0]} in {dt:.3f} s, "
          f"{rays / dt / 1e6:.1f} Mrays/s")
    del keep
    return 0


if __name__ == "__main__":
    sys.exit(main())
