"""Build recipe for the test oracle (test infrastructure only).

Produces
  oracle/_build/libhea_oracle.so   the CPU restatement (hea_oracle.c), plain C
  oracle/_ref/libref_accelerate.so the reference CPU engine, compiled from the
                                   reference's own pyhea/cpp/accelerate.cpp with
                                   ref_harness.cpp and the single-rank MPI stub
  oracle/_ref/pymod/accelerate<ext> the reference's own pybind11 module (its
                                   pyhea/cpp/bind.cpp + accelerate.cpp, CPU engine
                                   only), for the test of the install layout that
                                   keeps `device: cpu` beside the drop-in

The reference tree is read in place from REFERENCE_ROOT: the environment
variable HEA_REFERENCE_ROOT, else a checkout named `reference` beside this
repository; its sources are never copied.  When the tree is absent (as on
a machine that only runs the prebuilt files) the reference library is left as
it is.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE_ROOT = os.environ.get("HEA_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                                      "reference")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_oracle():
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libhea_oracle.so")
    src = os.path.join(HERE, "hea_oracle.c")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    # -ffp-contract=off: every fused multiply-add in the fitness is an explicit fma()
    _run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", src, "-o", out, "-lm"])
    return out


def build_reference():
    src_dir = os.path.join(REFERENCE_ROOT, "pyhea", "cpp")
    if not os.path.exists(os.path.join(src_dir, "accelerate.cpp")):
        return None
    out_dir = os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libref_accelerate.so")
    harness = os.path.join(HERE, "ref_harness.cpp")
    deps = [harness, os.path.join(src_dir, "accelerate.cpp"), os.path.join(HERE, "mpi_stub", "mpi.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    # the same flags the reference build uses for its CPU engine (C++14, -O3);
    # <tuple> is included by the harness because accelerate.cpp uses
    # std::make_tuple without including it
    _run(["g++", "-O3", "-std=c++14", "-fPIC", "-shared", "-I", os.path.join(HERE, "mpi_stub"), "-I", src_dir,
          harness, "-o", out, "-Wl,-Bsymbolic-functions", "-ldl"])
    return out


def build_reference_module():
    """PyHEA's own `accelerate` extension module as its build makes it for the CPU engine
    (bind.cpp + accelerate.cpp, no USE_CUDA), with the single-rank MPI stub."""
    import sysconfig

    src_dir = os.path.join(REFERENCE_ROOT, "pyhea", "cpp")
    if not os.path.exists(os.path.join(src_dir, "bind.cpp")):
        return None
    out_dir = os.path.join(HERE, "_ref", "pymod")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "accelerate" + sysconfig.get_config_var("EXT_SUFFIX"))
    srcs = [os.path.join(src_dir, "bind.cpp"), os.path.join(src_dir, "accelerate.cpp")]
    deps = srcs + [os.path.join(HERE, "mpi_stub", "mpi.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    import pybind11

    _run(["g++", "-O3", "-std=c++14", "-fPIC", "-shared", "-include", "tuple", "-I", os.path.join(HERE, "mpi_stub"),
          "-I", src_dir, "-I", sysconfig.get_paths()["include"], "-I", pybind11.get_include(), *srcs, "-o", out])
    return out


if __name__ == "__main__":
    print(build_oracle())
    print(build_reference_module() or "reference tree not found; oracle/_ref/pymod left as is")
    r = build_reference()
    print(r if r else "reference tree not found; oracle/_ref left as is")
    sys.exit(0)
