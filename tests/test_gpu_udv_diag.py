"""UDV scale diagnostics (udv_scale_file / udv_centered_file) on the GPU.

Records are taken where the reference takes them (src/green.c:214,238;
src/dqmc.c:707,772,831,926) and written in its formats (src/dqmc.c:158-340).
The values are statistics of this engine's own factors: its QR sorts columns
by norm first, the reference's dgeqrf does not, so log|D| of the same
product differ between the two by up to a few units.  Hence the pins:

* record structure line for line against the reference program (which
  factor, sweep count, tau, boundary, direction, entry counts);
* the first non-trivial suffix-stack record of a sweep is the factor of one
  block product B(b_M, b_{M-1}) of the current field: its log|D| extremes
  equal numpy's |diag R| of that product with its columns sorted by norm
  (1e-10);
* internal relations of each line (spread, cross, centered radius, offset).
"""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")

EXE = os.path.join(PKG, "dqmc_gpu")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "dqmc")

BASE = """lattice=square
Lx=4
Ly=4
pbc=1
t=-1.0
U=4.0
dtau=0.1
beta_list=2.0,4.0
nwarm=3
nmeas=4
nbin=2
nrep=2
seed=3
stab=8
"""


def rows(path):
    return [l.split() for l in open(path) if not l.startswith("#")]


def run(exe, d, text):
    d.mkdir(parents=True, exist_ok=True)
    (d / "input.txt").write_text(text)
    r = subprocess.run([exe, "input.txt"], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return d


def fnan(x):
    v = float(x)
    return v


def check_scale_line(x):
    lmin, lmax, lsp = fnan(x[12]), fnan(x[13]), fnan(x[14])
    rmin, rmax, rsp = fnan(x[18]), fnan(x[19]), fnan(x[20])
    assert math.isclose(lsp, lmax - lmin, rel_tol=0, abs_tol=1e-12)
    if x[11] in ("forward", "backward"):
        assert math.isclose(rsp, rmax - rmin, rel_tol=0, abs_tol=1e-12)
        assert math.isclose(fnan(x[24]), lmax + rmax, rel_tol=0, abs_tol=1e-12)
    else:   # single-factor sentinel (tests/test_dqmc.c:69-77)
        assert math.isnan(rmin) and math.isnan(rmax) and math.isnan(rsp)
        assert x[21:24] == ["0", "0", "0"] and math.isnan(fnan(x[24]))


@pytest.mark.parametrize("extra", ["", "sweep_order=alternating\n"])
def test_scale_file_structure_matches_reference(tmp_path, extra):
    if not os.path.exists(REF_EXE):
        pytest.skip("reference program not built here")
    text = BASE + extra + "udv_scale_file=udv_scale.dat\n"
    g = run(EXE, tmp_path / "gpu", text)
    r = run(REF_EXE, tmp_path / "ref", text)
    hg = open(g / "udv_scale.dat").readline()
    assert hg == open(r / "udv_scale.dat").readline()
    a, b = rows(g / "udv_scale.dat"), rows(r / "udv_scale.dat")
    assert len(a) == len(b) > 0
    for x, y in zip(a, b):
        assert len(x) == len(y) == 25
        assert x[:12] == y[:12]                       # metadata, sweep, tau, boundary, direction
        assert x[15:18] == y[15:18] and x[21:24] == y[21:24]   # entry counts
        check_scale_line(x)
    # the observables of the run are unaffected by recording
    obs = [l for l in open(g / "observables.dat") if not l.startswith("#")]
    plain = run(EXE, tmp_path / "plain", BASE + extra)
    assert obs == [l for l in open(plain / "observables.dat") if not l.startswith("#")]


def test_centered_file_structure_matches_reference(tmp_path):
    if not os.path.exists(REF_EXE):
        pytest.skip("reference program not built here")
    text = BASE + "green_rebuild=centered\nudv_centered_file=udv_centered.dat\n"
    g = run(EXE, tmp_path / "gpu", text)
    r = run(REF_EXE, tmp_path / "ref", text)
    assert open(g / "udv_centered.dat").readline() == open(r / "udv_centered.dat").readline()
    a, b = rows(g / "udv_centered.dat"), rows(r / "udv_centered.dat")
    assert len(a) == len(b) > 0
    for x, y in zip(a, b):
        assert len(x) == len(y) == 18
        assert x[:9] == y[:9]
        assert x[16:] == y[16:] == ["0", "ok"]
        smin, smax, rad, off, emin, emax, margin = (float(v) for v in x[9:16])
        assert math.isclose(rad, 0.5 * (emax - emin), abs_tol=1e-12)
        assert math.isclose(smin, emin - off, abs_tol=1e-12)
        assert math.isclose(smax, emax - off, abs_tol=1e-12)
        assert math.isclose(margin, math.log(np.finfo(float).max) - rad, abs_tol=1e-9)


def test_stack_record_equals_sorted_qr_of_block_product():
    Lx, U, dtau, L, stab, seed = 4, 4.0, 0.1, 20, 5, 9
    T, bp = dq.square_lattice(Lx, Lx)
    eng = dq.Engine(udv_diag=1)
    m = eng.add_model(T, bp, U, dtau, Lx, Lx)
    eng.add_chain(m, L, stab, seed)
    eng.prepare(1)
    n = Lx * Lx
    field = eng.field(0).reshape(L, n)
    eng.sweep(1)
    rec = eng.udv_records(0)
    M = L // stab
    kinds = [dq.UDV_DIRECTIONS[int(k)] for k in rec[:, 0]]
    assert kinds == ["stack_suffix_pre_rmul"] * (M - 1) + ["forward"] * (M - 1) + \
        ["left_udv_forward"]
    assert list(rec[: M - 1, 2]) == list(range(M - 1, 0, -1))
    assert all(rec[:, 3] == 0)                          # sweep_count before the increment
    np.testing.assert_array_equal(rec[0, 4:9], [0, 0, n, 0, 0])   # identity factor
    # B(b_M, b_{M-1}) = B_{L-1} ... B_{L-stab}, B_l = expK diag(exp(lambda s - dtau U / 2))
    K = T - (U / 2) * np.eye(n)
    w, V = np.linalg.eigh(K)
    expK = (V * np.exp(-dtau * w)) @ V.T
    lam = math.acosh(math.exp(dtau * U / 2))
    P = np.eye(n)
    for l in range(L - stab, L):
        P = expK @ np.diag(np.exp(lam * field[l] - dtau * U / 2)) @ P
    order = np.argsort(-np.linalg.norm(P, axis=0), kind="stable")
    ell = np.log(np.abs(np.diag(np.linalg.qr(P[:, order])[1])))
    assert abs(rec[1, 4] - ell.min()) < 1e-10 and abs(rec[1, 5] - ell.max()) < 1e-10
    assert list(rec[1, 6:9]) == [n, 0, 0]
    # records of later sweeps carry their sweep count; reading drains them
    eng.sweep(2)
    again = eng.udv_records(0)
    assert sorted(set(again[:, 3])) == [1, 2]
    assert len(eng.udv_records(0)) == 0
    eng.close()


def test_records_need_the_flag():
    T, bp = dq.square_lattice(4, 4)
    eng = dq.Engine()
    m = eng.add_model(T, bp, 4.0, 0.1, 4, 4)
    eng.add_chain(m, 10, 5, 1)
    eng.prepare(1)
    with pytest.raises(dq.DqmcError):
        eng.udv_records(0)
    eng.close()
