"""C ABI checks that need no GPU: the library loads, exports every symbol
include/*.h declares, host helpers compute what the reference computes, and
device calls fail loudly (no CPU fallback) when no GPU is present."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden, have_gpu, rel_err

dq = pytest.importorskip("dqmc_b200")


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(dqmc_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    lib = C.CDLL(dq.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_expm_matches_reference_model():
    for name in ("chain4_b2", "sq6_b2"):
        g = golden(name)
        n = g["thop"].shape[0]
        K = g["thop"] - float(g["U"]) / 2 * np.eye(n)
        assert rel_err(dq.expm_sym(K, -float(g["dtau"])), g["expK"]) < 1e-13
        assert rel_err(dq.expm_sym(K, float(g["dtau"])), g["expKinv"]) < 1e-13


def test_expm_edge_cases():
    """The host eigensolver behind the model exponential (Householder
    tridiagonalization + implicit symmetric QR): sizes 1 and 2, a dense
    random symmetric matrix, and a spectrum with repeated eigenvalues, each
    against numpy's eigh; expK expK^-1 = I."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((50, 50))
    blocks = np.kron(np.eye(5), np.ones((4, 4))) - 2.0 * np.eye(20)   # eigenvalues 2, -2 repeated
    for K in (np.array([[0.7]]), np.array([[1.0, -0.5], [-0.5, 3.0]]), A + A.T, blocks,
              np.zeros((6, 6))):
        for sc in (-0.1, 0.25):
            w, V = np.linalg.eigh(K)
            want = (V * np.exp(sc * w)) @ V.T
            got = dq.expm_sym(K, sc)
            assert np.max(np.abs(got - want)) < 1e-12 * max(1.0, np.max(np.abs(want)))
        E = dq.expm_sym(K, -0.1) @ dq.expm_sym(K, 0.1)
        assert np.max(np.abs(E - np.eye(K.shape[0]))) < 1e-12


def test_lattices_match_reference():
    for name in ("chain4_b2", "sq4_b4", "sq8_b4"):
        g = golden(name)
        kind, Lx, Ly = (int(x) for x in g["params"][:3])
        T, bp = dq.chain_lattice(Lx) if kind == 0 else dq.square_lattice(Lx, Ly)
        np.testing.assert_array_equal(T, g["thop"])
        np.testing.assert_array_equal(bp, g["bipart"])


@pytest.mark.skipif(have_gpu(), reason="checks the no-GPU error path")
def test_engine_fails_loudly_without_gpu():
    with pytest.raises(dq.DqmcError, match="no CUDA device"):
        dq.Engine()
    with pytest.raises(dq.DqmcError):
        g = golden("udv_fixture")
        dq.udv_green(g["U"], g["D"], g["T"])
