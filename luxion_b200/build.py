"""Build libluxion.so (the C-ABI library) in-tree for sm_100a.

    python -m luxion_b200.build            # build if sources changed
    python -m luxion_b200.build --force

Translation units:
  trace.cu    traversal kernels, FMA contraction on (exact steps use __f*_rn intrinsics)
  shade.cu    camera / shade / accumulate kernels, --fmad=false so every float op is
              rounded on its own, in the reference's order
  sort.cu     Morton keys and the radix sort of a bounce queue
  trace_static.cu  the fixed device scratch of lux_trace_rays_static
  texconv.cu  texel conversion (8/16-bit to float or binary16) at scene upload
  bvh_gpu.cu  device BVH8 build (binned SAH + collapse) and scene-geometry kernels,
              --fmad=false so every step rounds as the host builder's does
  context.cpp, engine.cpp, geometry.cpp, bvh_build.cpp, scene_gen.cpp   host C++ (no FMA contraction)
The CUDA runtime is linked statically so the library does not depend on which libcudart a
host process (for example PyTorch) has already loaded.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libluxion.so")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_UNITS = {
    "trace.cu": ["--fmad=true"],
    "shade.cu": ["--fmad=false"],
    "sort.cu": ["--fmad=true"],
    "trace_static.cu": ["--fmad=true"],
    "bvh_gpu.cu": ["--fmad=false"],
    "texconv.cu": ["--fmad=false"],
}
CPP_UNITS = ["context.cpp", "engine.cpp", "geometry.cpp", "bvh_build.cpp", "scene_gen.cpp"]


def _sources():
    files = sorted(f for f in os.listdir(CSRC) if not f.startswith("."))
    return [os.path.join(CSRC, f) for f in files] + [os.path.join(INCLUDE, "luxion.h"), __file__]


def _digest() -> str:
    h = hashlib.sha256()
    for p in _sources():
        with open(p, "rb") as f:
            h.update(os.path.basename(p).encode())
            h.update(f.read())
    return h.hexdigest()


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    stamp = os.path.join(OUT, "build.sha256")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}; cannot build the CUDA library")
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    common = ["-std=c++17", "-O3", "-I" + INCLUDE, "-I" + CSRC]
    jobs = []
    for unit, extra in CU_UNITS.items():
        obj = os.path.join(objdir, unit + ".o")
        jobs.append([NVCC, *ARCH, "-lineinfo", *common, *extra, "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "-Xptxas", "-v", "-c", os.path.join(CSRC, unit), "-o", obj])
    gxx = shutil.which("g++") or "g++"
    for unit in CPP_UNITS:
        obj = os.path.join(objdir, unit + ".o")
        jobs.append([gxx, *common, "-fPIC", "-ffp-contract=off", "-I" + os.path.join(CUDA_HOME, "include"),
                     "-c", os.path.join(CSRC, unit), "-o", obj])
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
        for out in ex.map(_run, jobs):
            logs.append(out)
    objs = [os.path.join(objdir, u + ".o") for u in list(CU_UNITS) + CPP_UNITS]
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lpthread"])
    os.replace(tmp, LIB)
    with open(os.path.join(OUT, "ptxas.log"), "w") as f:
        f.write("\n".join(logs))
    with open(stamp, "w") as f:
        f.write(dig)
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
