"""The reference-side binding (luxion_b200/shim/pathtrace_luxion.cpp) compiles against the
reference's own headers and links against libluxion with every symbol resolved.

The shim defines pathtraceInit / pathtrace / pathtraceFree / copyImageToHost with the
reference's signatures (checked by static_asserts against include/pathtrace.h and
include/pathtrace/pathtrace_buffers.h of the reference). The reference's headers are CUDA
C++; they are compiled for the host here with the same force-included prelude and stubs the
oracle's reference build uses (oracle/ref/prelude.h, oracle/ref/stub). Skipped where the
reference checkout (beside this repository) is absent."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("LUXION_REFERENCE", os.path.normpath(os.path.join(ROOT, "..", "reference")))
SHIM = os.path.join(ROOT, "luxion_b200", "shim", "pathtrace_luxion.cpp")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include")), reason="reference checkout absent")
def test_shim_compiles_against_reference_headers_and_links(tmp_path):
    import luxion_b200 as lx
    lx.lib()  # builds libluxion.so if needed
    import torch
    fmt = os.path.join(os.path.dirname(torch.__file__), "include")
    obj = str(tmp_path / "shim.o")
    cmd = ["g++", "-std=c++17", "-fPIC", "-w", "-c", "-include", os.path.join(ROOT, "oracle", "ref", "prelude.h"),
           "-D__device__=", "-D__host__=", "-D__global__=", "-D__constant__=",
           "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_CPP", "-DFMT_HEADER_ONLY",
           "-I" + os.path.join(ROOT, "oracle", "ref", "stub"), "-I" + os.path.join(REF, "include"),
           "-I" + os.path.join(REF, "src"), "-I" + os.path.join(REF, "external", "include"),
           "-I" + os.path.join(CUDA, "include"), "-I" + fmt, "-I" + os.path.join(ROOT, "include"),
           "-x", "c++", SHIM, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    so = str(tmp_path / "libshim.so")
    link = ["g++", "-shared", "-o", so, obj, "-Wl,--no-undefined",
            "-L" + os.path.join(ROOT, "luxion_b200", "_lib"), "-lluxion",
            "-L" + os.path.join(CUDA, "lib64"), "-lcudart"]
    r = subprocess.run(link, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    nm = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
    for sym in ("_Z13pathtraceInitP5Scene", "_Z9pathtraceP6uchar4ii", "_Z13pathtraceFreev", "_Z15copyImageToHostv"):
        assert sym in nm, sym
