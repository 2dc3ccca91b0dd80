"""Pins the CPU oracle (oracle/oracle.c) to the reference's own outputs.

The golden .npz files were produced by the unmodified reference
(tests/golden/make_golden.py); the UDV fixture is the reference's
tests/fixtures/udv_phase6a_actual_n16*.txt re-packed.  Tolerances follow the
reference's tests: G 1e-9 (test_dqmc_stack.c:117-118), fixtures 1e-9
relative (test_udv_phase6a_fixture.c:130), field flips and counters exact.
"""
import numpy as np
import pytest

from conftest import CASES, case_args, golden, rel_err


def test_rng_streams_bit_exact(oracle):
    g = golden("rng")
    for s, d in zip(g["seeds"], g["draws"]):
        np.testing.assert_array_equal(oracle.rng(int(s), 16), d)
    for args, want in zip(g["replica_args"], g["replica_seeds"]):
        assert oracle.replica_seed(*(int(a) for a in args)) == int(want)
    m, e = oracle.jackknife(g["jk_x"])
    assert m == g["jk"][0] and abs(e - g["jk"][1]) < 1e-15


def test_jackknife_known_answer(oracle):
    # test_measure.c: jackknife of {1,3,5} = (3, sqrt(4/3))
    m, e = oracle.jackknife(np.array([1.0, 3.0, 5.0]))
    assert m == 3.0 and abs(e - np.sqrt(4.0 / 3.0)) < 1e-14


@pytest.mark.parametrize("name", CASES)
def test_model_and_green(oracle, name):
    g = golden(name)
    a = case_args(g)
    ch = oracle.chain(a["kind"], a["Lx"], a["Ly"], a["U"], a["dtau"], a["L"],
                      a["stab"], a["seed"])
    m = oracle.model(ch)
    np.testing.assert_array_equal(m["thop"], g["thop"])
    np.testing.assert_array_equal(m["bipart"], g["bipart"])
    assert rel_err(m["expK"], g["expK"]) < 1e-13
    assert rel_err(m["expKinv"], g["expKinv"]) < 1e-13
    st = ch.state()
    np.testing.assert_array_equal(st["field"], g["field0"])
    assert rel_err(st["Gu"], g["G0"]) < 1e-10
    rc, gs, ds = ch.green_scratch(0)
    assert rc == 0 and ds == int(g["det_sign"])
    assert rel_err(gs, g["G_scratch"]) < 1e-10
    assert rel_err(ch.wrap(0, g["G0"]), g["G_wrap0"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_sweeps_match_reference(oracle, name):
    g = golden(name)
    a = case_args(g)
    ch = oracle.chain(a["kind"], a["Lx"], a["Ly"], a["U"], a["dtau"], a["L"],
                      a["stab"], a["seed"], drift=True)
    sel = 2 if a["selector"] == "all" else 1
    for s in range(a["sweeps"]):
        ch.sweep(1)
        st = ch.state()
        np.testing.assert_array_equal(st["field"], g["fields"][s])
        att, acc, sw, status = (int(x) for x in g["counters"][s])
        assert (st["attempts"], st["accepted"], st["sweeps"], st["status"]) == \
            (att, acc, sw, status)
        assert np.max(np.abs(st["Gu"] - g["Gs"][s])) < 1e-9
        meas, szz, sperp = oracle.measure(ch, sel)
        assert np.max(np.abs(meas - g["meas"][s])) < 1e-9
        assert np.max(np.abs(szz - g["szz"][s])) < 1e-9
        assert np.max(np.abs(sperp - g["sperp"][s])) < 1e-9
    np.testing.assert_array_equal(ch.state()["rng"], g["rng_end"])
    # the drift maximum is rounding noise; bound it as test_dqmc_stab_drift.c
    # does (< 1e-6 up to U = 12) and require the same sample count
    d = oracle.drift(ch)
    assert d[0] == g["drift"][0]
    assert d[1] < 1e-6 and g["drift"][1] < 1e-6


def test_udv_fixture(oracle):
    g = golden("udv_fixture")
    assert abs(g["max_logD"] - g["min_logD"] - 1350.7731737311086) < 1e-9
    rc, G, ds = oracle.udv_inv(g["U"], g["D"], g["T"])
    assert rc == 0 and ds == int(g["det_sign"])
    assert rel_err(G, g["G"]) <= 1e-9


def test_u0_free_fermion_energy(oracle):
    # test_integration.c:88-169: at U = 0, E = 2 sum_k eps_k f(eps_k) with
    # mu = 0, and Szz(q) = sum_k f_k (1 - f_{k+q}) / (2 n), Sperp = 2 Szz.
    L, dtau = 20, 0.1
    beta = L * dtau
    ch = oracle.chain(0, 4, 1, 0.0, dtau, L, 8, 5)
    meas, szz, sperp = oracle.measure(ch, 2)
    k = 2 * np.pi * np.arange(4) / 4
    eps = -2.0 * np.cos(k)
    f = 1.0 / (np.exp(beta * eps) + 1.0)
    assert abs(meas[0] - 2.0 * np.sum(eps * f)) < 1e-7
    exact = np.array([np.sum(f * (1 - np.roll(f, -q))) / 8.0 for q in range(4)])
    assert np.max(np.abs(szz - exact)) < 1e-8
    assert np.max(np.abs(sperp - 2 * szz)) < 1e-12
