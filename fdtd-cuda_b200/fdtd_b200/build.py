"""Builds libfdtd_b200.so (the CUDA kernels and the C ABI) for sm_100a, and
fdtd_runner, the reference's program as a C++ host over that ABI.

Both are built in-tree next to this file so that they travel with the
repository; nvcc cross-compiles without a GPU.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")
LIB = os.path.join(HERE, "libfdtd_b200.so")
RUNNER = os.path.join(HERE, "fdtd_runner")
SOURCES = ["fdtd.cu", "setup.cpp"]
# -fmad=false: no multiply-add contraction chosen by the compiler.  A kernel
# body shared by two launch forms (one simulation, a batch) then rounds the
# same in both, and the arithmetic follows the order written, as in the FP64
# oracle (built with -ffp-contract=off).  The Yee passes spell their fused
# multiply-adds out with intrinsics, which this flag does not touch.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2", "-shared", "--expt-relaxed-constexpr", "-fmad=false",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    out = [os.path.join(CSRC, s) for s in SOURCES]
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "fdtd_b200.h"))
    return out, deps


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    _, deps = sources()
    return any(os.path.getmtime(d) > t for d in deps)


def build_runner(verbose=False):
    """fdtd_runner: host C++ only, linked against the library found next to
    it at run time."""
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", os.path.join(CSRC, "runner.cpp"),
           "-L" + HERE, "-lfdtd_b200", "-Wl,-rpath,$ORIGIN", "-o", RUNNER + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(RUNNER + ".tmp", RUNNER)
    return RUNNER


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build() and os.path.exists(RUNNER):
        return LIB
    srcs, _ = sources()
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", LIB + ".tmp", *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    build_runner(verbose)
    return LIB


if __name__ == "__main__":
    import sys
    build(force=True, verbose=True, extra=sys.argv[1:])
