"""Failure detection and resume, exercised from the host (no GPU fault).

A chain whose state is corrupted (non-finite G written from the host, as the
reference's own tests corrupt D.Gu.g) stops at its next stabilization point
with a sticky status and sign 0, and stays frozen; the other chains of the
same launch continue exactly as in a clean run.  A UDV with a non-finite
entry gives det sign 0.  Resuming a chain from its saved field and RNG state
continues the trajectory an uninterrupted run takes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")

ST_NONFINITE = 1


def batch(seeds, Lx=6, L=20, stab=8):
    T, bp = dq.square_lattice(Lx, Lx)
    e = dq.Engine()
    m = e.add_model(T, bp, 4.0, 0.1, Lx, Lx)
    for s in seeds:
        e.add_chain(m, L, stab, s)
    e.prepare(1)
    return e


def test_corrupted_chain_is_frozen_others_continue():
    seeds = [3, 4, 5]
    clean, hit = batch(seeds), batch(seeds)
    G = hit.green(1)
    G[2, 3] = np.nan
    hit.write_green(1, G)
    clean.sweep(2)
    hit.sweep(2)
    c = hit.counters(1)
    assert c["status"] & ST_NONFINITE and c["sign"] == 0.0 and c["sweeps"] == 0
    frozen = hit.field(1)       # flips before the first stabilization point may stand
    for k in (0, 2):
        np.testing.assert_array_equal(hit.field(k), clean.field(k))
        a, b = hit.counters(k), clean.counters(k)
        assert (a["attempts"], a["accepted"], a["sweeps"], a["status"]) == \
            (b["attempts"], b["accepted"], b["sweeps"], b["status"])
        assert np.max(np.abs(hit.green(k) - clean.green(k))) == 0.0
    hit.sweep(2)                                               # stays frozen
    c2 = hit.counters(1)
    assert c2["status"] == c["status"] and c2["sweeps"] == 0 and c2["attempts"] == c["attempts"]
    np.testing.assert_array_equal(hit.field(1), frozen)
    assert c["attempts"] < 8 * 36 + 36                          # stopped within the first block
    clean.close()
    hit.close()


def test_udv_green_nonfinite_input_gives_zero_sign():
    rng = np.random.default_rng(2)
    n = 8
    U, _ = np.linalg.qr(rng.standard_normal((n, n)))
    D = np.exp(rng.uniform(-5, 5, n))
    T = np.triu(rng.standard_normal((n, n)), 1) + np.eye(n)
    D[3] = np.nan
    G, ds = dq.udv_green(U, D, T)
    assert ds == 0


def test_resume_from_field_and_rng_continues_trajectory():
    seeds = [7, 8]
    whole = batch(seeds)
    whole.sweep(4)
    first = batch(seeds)
    first.sweep(2)
    saved = [(first.field(c), first.counters(c)["rng"]) for c in range(2)]
    first.close()
    second = batch(seeds)
    for c, (f, r) in enumerate(saved):
        second.write_field(c, f)
        second.write_rng(c, r)
    second.sweep(2)
    for c in range(2):
        np.testing.assert_array_equal(second.field(c), whole.field(c))
        np.testing.assert_array_equal(second.counters(c)["rng"], whole.counters(c)["rng"])
        assert np.max(np.abs(second.green(c) - whole.green(c))) < 1e-9
    whole.close()
    second.close()
