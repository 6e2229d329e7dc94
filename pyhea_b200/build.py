"""Build recipe of the product libraries (in-tree, sm_100a).

  pyhea_b200/libhea_cuda.so         kernels + C ABI (include/hea_cuda.h), nvcc
  pyhea_b200/accelerate<ext-suffix> pybind11 module `accelerate`, the drop-in for
                                    pyhea.cpp.accelerate; links libhea_cuda.so

Run `python pyhea_b200/build.py` (or __graft_entry__.build()).  Objects are
rebuilt when a source is newer than the library.
"""
import glob
import os
import subprocess
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(REPO, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIB = os.path.join(PKG, "libhea_cuda.so")
EXT = os.path.join(PKG, "accelerate" + sysconfig.get_config_var("EXT_SUFFIX"))


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_lib(verbose_ptxas=False):
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = cu + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if not _newer(LIB, deps) and not verbose_ptxas:
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I", INCLUDE, "-I", CSRC,
           "--expt-relaxed-constexpr", "-o", LIB, *cu]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    _run(cmd)
    return LIB


def build_ext():
    src = os.path.join(CSRC, "bind.cpp")
    if not _newer(EXT, [src, LIB, os.path.join(INCLUDE, "hea_cuda.h")]):
        return EXT
    import pybind11

    py_inc = sysconfig.get_paths()["include"]
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", "-I", py_inc, "-I",
          pybind11.get_include(), "-I", INCLUDE, src, "-o", EXT, "-L", PKG, "-lhea_cuda", "-Wl,-rpath,$ORIGIN"])
    return EXT


def build(verbose_ptxas=False):
    build_lib(verbose_ptxas)
    build_ext()
    return LIB, EXT


if __name__ == "__main__":
    import sys

    build(verbose_ptxas="-v" in sys.argv)
