"""Build recipe of the native library (nvcc for sm_100a + g++ for the C++ API).

Produces, in-tree so the files travel with the repository snapshot:

* ``spectral_upcxx_b200/lib/libspectral_b200.so`` -- the CUDA kernels, the
  C-ABI of ``include/spectral_b200.h`` and the C++ field API
  (``api/*.cpp``: Scalar, Vector, Operators, FFT1D, Writer, Particle).
* ``build_cpp_program(src, out)`` links a C++ program written against the
  reference's headers (DataObjects.H, Writer.H, ...) to that library.

Objects are rebuilt only when a source or header is newer than its output.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
API = os.path.join(PKG, "api")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIBNAME = "libspectral_b200.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-variable"]


def _cuda_home() -> str:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build spectral_upcxx_b200")


def _nvcc() -> str:
    return os.path.join(_cuda_home(), "bin", "nvcc")


def _cxx() -> str:
    # the system compiler; some environments point CXX at a wrapper without OpenMP
    return shutil.which("g++") or "g++"


def _newer(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def build_library(verbose: bool = False) -> str:
    """Compile and link libspectral_b200.so; returns its path."""
    os.makedirs(OBJDIR, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(API, "*.cpp")))
    cu_hdr = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [os.path.join(INCLUDE, "spectral_b200.h")]
    api_hdr = sorted(glob.glob(os.path.join(API, "*.H"))) + sorted(
        glob.glob(os.path.join(API, "upcxx", "*.hpp"))) + [os.path.join(INCLUDE, "spectral_b200.h")]
    jobs = []
    objs = []
    for src in cu:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(obj, [src] + cu_hdr):
            jobs.append([_nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-c", src, "-o", obj])
    cuda_inc = os.path.join(_cuda_home(), "include")
    for src in cpp:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(obj, [src] + api_hdr):
            jobs.append([_cxx()] + CXX_FLAGS + ["-I", API, "-I", INCLUDE, "-I", cuda_inc, "-c", src,
                                                "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            for out in ex.map(_run, jobs):
                if verbose and out:
                    print(out)
    if _newer(LIBPATH, objs) or jobs:
        _run([_nvcc()] + ARCH + ["-shared", "-o", LIBPATH] + objs + ["-lcudart_static", "-lrt",
                                                                     "-ldl", "-lpthread"])
    return LIBPATH


def build_cpp_program(sources, out: str, extra_flags=None) -> str:
    """Link a C++ program written against the reference API headers."""
    if not os.path.exists(LIBPATH):
        build_library()
    srcs = [sources] if isinstance(sources, str) else list(sources)
    # the API headers fix the class layouts the program is compiled against
    deps = srcs + [LIBPATH] + sorted(glob.glob(os.path.join(API, "*.H"))) + sorted(
        glob.glob(os.path.join(API, "upcxx", "*.hpp")))
    if _newer(out, deps):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        cmd = [_cxx(), "-O2", "-std=c++17", "-w", "-DDIM=3", "-I", API, "-I", INCLUDE] + (
            extra_flags or []) + srcs + ["-L", LIBDIR, "-lspectral_b200", f"-Wl,-rpath,{LIBDIR}",
                                         "-o", out]
        _run(cmd)
    return out


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv))
