"""Build the engine's native artefacts in-tree with nvcc (sm_100a only).

  pbbperm_b200/libpbbperm.so   kernels + host engine + C ABI (include/pbbperm.h)
  pbbperm_b200/bb              drop-in command line (`bb -z p=fsp,i=...`)
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpbbperm.so")
CLI = os.path.join(PKG, "bb")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]

LIB_SOURCES = ["pbb_kernels.cu", "pbb_host.cu", "pbb_diag.cu", "pbb_noalloc.cu", "pbb_pool.cu", "pbb_heur.cu",
               "pbb_ckpt.cu"]
LIB_DEPS = LIB_SOURCES + ["pbb_types.h", "pbb_device.cuh", "pbb_launch.h", "pbb_tables.h", "pbb_heur.h",
                          "pbb_devguard.h"]
HEADERS = ["pbbperm.h", "pbbperm_diag.h"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    deps = [os.path.join(CSRC, f) for f in LIB_DEPS] + [os.path.join(ROOT, "include", h) for h in HEADERS]
    if force or _stale(LIB, deps):
        cmd = [_nvcc()] + NVFLAGS + ["-shared", "-o", LIB] + [os.path.join(CSRC, f) for f in LIB_SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    cli_src = os.path.join(CSRC, "bb_main.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB, os.path.join(CSRC, "ini.h")])):
        cmd = ["g++", "-O2", "-std=c++17", "-o", CLI, cli_src, "-I", os.path.join(ROOT, "include"),
               "-L", PKG, "-lpbbperm", "-Wl,-rpath,$ORIGIN", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
