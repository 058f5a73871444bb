"""Build recipe for the CPU oracle and the reference-side checkers.

TEST INFRASTRUCTURE ONLY.  Produces
  oracle/liboracle.so         -- the C++ restatement (oracle.hpp), IEEE float,
                                 no FMA contraction, std::thread loops
  oracle/_ref/libref_host.so  -- the REFERENCE's own __host__ __device__ code
                                 compiled for the host from the sources where
                                 they lie (only when the reference tree is
                                 present; the built file is git-ignored and
                                 travels with the working tree)

Usage: python oracle/build_oracle.py [--reference-root PATH] [--force]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# where the reference's source tree lies in the build container; the
# CUPBR_REFERENCE_ROOT environment variable points the recipe elsewhere
DEFAULT_REF = os.environ.get("CUPBR_REFERENCE_ROOT", "/root/reference")
CUDA_INC = "/usr/local/cuda/include"

CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-ffp-contract=off", "-fno-fast-math",
            "-D_USE_MATH_DEFINES"]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_oracle(force: bool = False) -> str:
    out = os.path.join(HERE, "liboracle.so")
    srcs = [os.path.join(HERE, "oracle_capi.cpp"), os.path.join(HERE, "oracle.hpp")]
    if force or _newer(out, srcs):
        _run(["g++", *CXXFLAGS, srcs[0], "-o", out])
    return out


def build_ref_host(ref_root: str, force: bool = False) -> str | None:
    """Compile the reference's host-callable code plus oracle/ref_host.cpp."""
    lib_inc = os.path.join(ref_root, "lib", "include")
    if not os.path.isdir(lib_inc):
        return None
    outdir = os.path.join(HERE, "_ref")
    os.makedirs(outdir, exist_ok=True)
    stub = os.path.join(outdir, "stub_include", "GLFW")
    os.makedirs(stub, exist_ok=True)
    # Camera.h includes GLFW for its input handler only; a forward declaration
    # is all the pose accessors need.
    with open(os.path.join(stub, "glfw3.h"), "w") as f:
        f.write("#pragma once\ntypedef struct GLFWwindow GLFWwindow;\n")
    src = os.path.join(ref_root, "lib", "src")
    ref_units = [os.path.join(src, p) for p in (
        "Geometry/Geometry.cu", "Geometry/Triangle.cu", "Geometry/Sphere.cu", "Geometry/Quad.cu",
        "Geometry/Plane.cu", "Geometry/Mesh.cu", "DataStructure/BoundingVolumeHierarchy.cpp", "Core/Memory.cu")]
    mine = [os.path.join(HERE, "ref_host.cpp"), os.path.join(HERE, "cuda_host_shim.cpp")]
    out = os.path.join(outdir, "libref_host.so")
    if force or _newer(out, mine + ref_units + [os.path.join(HERE, "device_overloads.h")]):
        # -Bsymbolic: the reference's cudaMalloc / cudaMemcpy calls must bind
        # to the host shim in this library even when a real CUDA runtime
        # (e.g. PyTorch's) is already loaded into the process.
        _run(["g++", *CXXFLAGS, "-Wl,-Bsymbolic", "-w", "-include", "cstdint", "-include", "cstring", "-include",
              os.path.join(HERE, "device_overloads.h"), "-I", lib_inc,
              "-I", CUDA_INC, "-I", os.path.join(outdir, "stub_include"), *mine,
              "-x", "c++", *ref_units, "-o", out])
    return out


STB_WRITE_STUB = """#pragma once
/* ToneMapper.cu includes stb_image_write.h for saveToFile only; the
   submodule is empty in the reference tree and saveToFile is never called
   by the driver, so these two entry points are inert stand-ins. */
static inline void stbi_flip_vertically_on_write(int) {}
static inline int stbi_write_bmp(char const*, int, int, int, const void*) { return 0; }
"""


def build_ref_cuda(ref_root: str, force: bool = False) -> str | None:
    """Compile the reference's CUDA path for sm_100a (-use_fast_math, as its
    CMakeLists.txt:61) with oracle/ref_cuda.cu into oracle/_ref/libref_cuda.so."""
    lib_inc = os.path.join(ref_root, "lib", "include")
    if not os.path.isdir(lib_inc):
        return None
    outdir = os.path.join(HERE, "_ref")
    stub = os.path.join(outdir, "stub_include")
    os.makedirs(os.path.join(stub, "GLFW"), exist_ok=True)
    with open(os.path.join(stub, "GLFW", "glfw3.h"), "w") as f:
        f.write("#pragma once\ntypedef struct GLFWwindow GLFWwindow;\n")
    with open(os.path.join(stub, "stb_image_write.h"), "w") as f:
        f.write(STB_WRITE_STUB)
    src = os.path.join(ref_root, "lib", "src")
    ref_units = [os.path.join(src, p) for p in (
        "Renderer/PathTracer.cu", "Renderer/VolumeRenderer.cu", "Renderer/GradientDomain.cu",
        "Renderer/RayTracer.cu", "Geometry/Geometry.cu", "Geometry/Triangle.cu", "Geometry/Sphere.cu",
        "Geometry/Quad.cu", "Geometry/Plane.cu", "Geometry/Mesh.cu", "DataStructure/BoundingVolumeHierarchy.cpp",
        "Core/Memory.cu", "PostProcessing/PostProcessor.cpp", "PostProcessing/PyramidConstructor.cu",
        "PostProcessing/Convolution.cu", "Renderer/ToneMapper.cu")]
    mine = os.path.join(HERE, "ref_cuda.cu")
    out = os.path.join(outdir, "libref_cuda.so")
    if not (force or _newer(out, [mine] + ref_units)):
        return out
    objdir = os.path.join(outdir, "obj")
    os.makedirs(objdir, exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc"
    flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-use_fast_math", "-O3", "-std=c++17",
             "-D_USE_MATH_DEFINES", "-include", "cstdint", "-Xcompiler", "-fPIC", "-w", "-I", lib_inc, "-I", stub,
             "-I", CUDA_INC]
    jobs = [(s, os.path.join(objdir, f"{i:02d}_{os.path.basename(s)}.o")) for i, s in enumerate([mine] + ref_units)]
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        list(ex.map(lambda j: subprocess.check_call([nvcc, *flags, "-c", j[0], "-o", j[1]]), jobs))
    objs = [o for _, o in jobs]
    _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", out, *objs,
          "-Xlinker", "-Bsymbolic"])
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default=DEFAULT_REF)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build_oracle(a.force)
    r = build_ref_host(a.reference_root, a.force)
    print("ref_host:", r)
    print("ref_cuda:", build_ref_cuda(a.reference_root, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
