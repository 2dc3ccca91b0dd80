"""Build libdqmc_b200.so (sm_100a) and the dqmc_gpu command-line driver.

Everything is compiled in-tree with nvcc/gcc so the artefacts travel with
the source tree:

* ``sai-qmc_b200/libdqmc_b200.so`` -- CUDA kernels + host engine + C ABI
  (include/dqmc_gpu.h) + host driver library (include/dqmc_host.h)
* ``sai-qmc_b200/dqmc_gpu`` -- the C driver (``dqmc_gpu input.txt``)
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libdqmc_b200.so")
EXE = os.path.join(PKG, "dqmc_gpu")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    cu = sorted(glob.glob(os.path.join(PKG, "csrc", "*.cu")))
    hdr = sorted(glob.glob(os.path.join(PKG, "csrc", "*.cuh")) +
                 glob.glob(os.path.join(PKG, "csrc", "*.h")) +
                 glob.glob(os.path.join(ROOT, "include", "*.h")))
    host = sorted(glob.glob(os.path.join(PKG, "host", "*.c")))
    return cu, hdr, host


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    cu, hdr, host = _sources()
    lib_host = [h for h in host if not h.endswith("dqmc_main.c")]
    main = [h for h in host if h.endswith("dqmc_main.c")]
    if force or _stale(LIB, cu + hdr + lib_host):
        objs = []
        bdir = os.path.join(ROOT, "_build")
        os.makedirs(bdir, exist_ok=True)
        for src in lib_host:
            obj = os.path.join(bdir, os.path.basename(src) + ".o")
            subprocess.run(["gcc", "-std=c11", "-O2", "-fPIC", "-Wall", "-Wextra",
                            "-I", os.path.join(ROOT, "include"), "-c", src, "-o",
                            obj], check=True)
            objs.append(obj)
        # the CUDA translation units compile in parallel (each takes minutes)
        flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-I", os.path.join(ROOT, "include")]
        if verbose:
            flags.append("-Xptxas=-v")
        procs, cobjs = [], []
        for src in cu:
            obj = os.path.join(bdir, os.path.basename(src) + ".o")
            procs.append(subprocess.Popen([NVCC, *flags, "-c", src, "-o", obj]))
            cobjs.append(obj)
        if any([p.wait() != 0 for p in procs]):
            raise subprocess.CalledProcessError(1, "nvcc")
        subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *cobjs, *objs], check=True)
    if main and (force or _stale(EXE, main + [LIB] + hdr)):
        subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Wextra",
                        "-I", os.path.join(ROOT, "include"), "-o", EXE, *main,
                        "-L", PKG, "-ldqmc_b200", "-Wl,-rpath,$ORIGIN", "-lm"],
                       check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
