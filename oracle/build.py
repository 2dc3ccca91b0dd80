"""Build recipe for the CPU oracle (test infrastructure only).

Two artefacts:

* ``oracle/liboracle.so`` -- the plain-C restatement of the reference's BSS
  sweep in ``oracle/oracle.c`` (no external libraries; built everywhere).
* ``oracle/_ref/`` -- the UNMODIFIED reference compiled from its own sources
  where they lie (``$SAIQMC_REF``, else a ``reference`` directory beside
  the repository), linked
  against the OpenBLAS 0.3.15 that ships inside the opencv wheel of this
  image (the reference calls Fortran BLAS/LAPACK symbols, linalg.c:27-42):
    - ``libdqmcref.so``: reference src/*.c minus main.c + ``ref_shim.c``
    - ``dqmc``: the reference command-line program (CPU baseline)
  Nothing is copied out of the reference tree; objects go to ``_ref/`` only.

Run ``python oracle/build.py`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import glob
import os
import site
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: $SAIQMC_REF, else a "reference" directory beside
# the repository root.
REF = os.environ.get("SAIQMC_REF") or os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                  "reference")
OUT = os.path.join(HERE, "_ref")


def _run(cmd):
    subprocess.run(cmd, check=True)


def find_openblas():
    """Locate an LP64 OpenBLAS exporting plain dgemm_/dgeqrf_/... symbols."""
    roots = list(site.getsitepackages()) + [site.getusersitepackages()]
    for r in roots:
        hits = sorted(glob.glob(os.path.join(r, "opencv_python_headless.libs",
                                             "libopenblasp-*.so")))
        if hits:
            libdir = os.path.dirname(hits[0])
            extra = [os.path.join(r, "scipy.libs")]
            return hits[0], [libdir] + extra
    return None, []


def build_oracle():
    src = os.path.join(HERE, "oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if (os.path.exists(out)
            and os.path.getmtime(out) >= os.path.getmtime(src)):
        return out
    _run(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra",
          "-o", out, src, "-lm"])
    return out


def build_ref(force=False):
    """Compile the reference; returns the output dir or None if unavailable."""
    srcdir = os.path.join(REF, "src")
    if not os.path.isdir(srcdir):
        return None
    blas, rpaths = find_openblas()
    if blas is None:
        print("oracle/build.py: no OpenBLAS found; reference not built",
              file=sys.stderr)
        return None
    os.makedirs(OUT, exist_ok=True)
    lib = os.path.join(OUT, "libdqmcref.so")
    exe = os.path.join(OUT, "dqmc")
    shim = os.path.join(HERE, "ref_shim.c")
    if not force and os.path.exists(lib) and os.path.exists(exe) and \
            os.path.getmtime(lib) >= os.path.getmtime(shim):
        return OUT
    srcs = sorted(glob.glob(os.path.join(srcdir, "*.c")))
    lib_srcs = [s for s in srcs if os.path.basename(s) != "main.c"]
    ldflags = ([blas, "-Wl,--disable-new-dtags"]
               + [f"-Wl,-rpath,{p}" for p in rpaths] + ["-lm"])
    cflags = ["-std=c11", "-O2", "-I", srcdir, "-w"]
    _run(["gcc", *cflags, "-fPIC", "-shared", "-o", lib, shim, *lib_srcs,
          *ldflags])
    _run(["gcc", *cflags, "-o", exe, *srcs, *ldflags])
    return OUT


def main():
    print(build_oracle())
    print(build_ref(force="--force" in sys.argv))


if __name__ == "__main__":
    main()
