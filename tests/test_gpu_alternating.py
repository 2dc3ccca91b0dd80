"""sweep_order=alternating on the GPU vs the reference (golden vectors made
by the reference's own alternating sweeps, tests/golden/make_golden.py).

Forward sweeps store the prefix stack and reuse the suffix stack the
backward sweep before them rebuilt; backward sweeps wrap with B^-1 G B and
form G at each boundary from the carried prefix and the new suffix
(src/dqmc.c:609-963).  Same bars as the forward parity tests: field flips,
counters and RNG state bit-exact, G within 1e-9, reference-definition drift
with the same number of samples.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")

ALT_CASES = ["chain4_alt", "sq4_b4_alt", "sq6_b2_alt", "sq8_b4_alt"]


def alt_engine(g, delay_rank=0, drift=dq.DRIFT_STAB):
    kind, Lx, Ly, L, stab, seed, sweeps = (int(x) for x in g["params"])
    if kind == 0:
        T, bp = dq.chain_lattice(Lx)
        Ly = 1
    else:
        T, bp = dq.square_lattice(Lx, Ly)
    eng = dq.Engine(delay_rank=delay_rank, drift=drift, sweep_order=dq.SWEEP_ALTERNATING)
    m = eng.add_model(T, bp, float(g["U"]), float(g["dtau"]), Lx, Ly)
    eng.add_chain(m, L, stab, seed)
    eng.prepare(1)
    return eng, sweeps


@pytest.mark.parametrize("name", ALT_CASES)
@pytest.mark.parametrize("kb", [0, 5])
def test_alternating_matches_reference(name, kb):
    g = golden(name)
    eng, sweeps = alt_engine(g, delay_rank=kb)
    np.testing.assert_array_equal(eng.field(0), g["field0"])
    for s in range(sweeps):
        eng.sweep(1)
        np.testing.assert_array_equal(eng.field(0), g["fields"][s])
        c = eng.counters(0)
        att, acc, sw, status = (int(x) for x in g["counters"][s])
        assert (c["attempts"], c["accepted"], c["sweeps"], c["status"]) == (att, acc, sw, status)
        assert np.max(np.abs(eng.green(0) - g["Gs"][s])) < 1e-9, s
    np.testing.assert_array_equal(eng.counters(0)["rng"], g["rng_end"])
    eng.close()


def test_alternating_reference_drift():
    g = golden("sq6_b2_alt")
    eng, sweeps = alt_engine(g, drift=dq.DRIFT_STAB | dq.DRIFT_SCRATCH)
    eng.sweep(sweeps)
    c = eng.counters(0)
    assert c["scratch_drift_samples"] == int(g["drift"][0])
    assert c["scratch_drift_max"] < 1e-6 and c["drift_max"] < 1e-6
    assert c["drift_samples"] == c["scratch_drift_samples"]
    eng.close()


def test_alternating_headline_lattice_matches_reference():
    """16x16, U=4, beta=8, stab=8, the benchmark's replica seeds: over two
    forward and two backward sweeps every chain flips exactly the fields of
    the reference.  Chain 0's first backward sweep meets an acceptance
    decision at the rounding level (slice 17, site 236): the reference run
    with one BLAS thread and the same reference with 2, 4 or 8 threads take
    it opposite ways, so a chain must follow one of the two reference
    trajectories (fields, fields_t4) throughout."""
    g = golden("sq16_b8_alt")
    Lx, L, stab, sweeps = (int(x) for x in g["params"])
    T, bp = dq.square_lattice(Lx, Lx)
    eng = dq.Engine(drift=dq.DRIFT_STAB | dq.DRIFT_SCRATCH, sweep_order=dq.SWEEP_ALTERNATING)
    m = eng.add_model(T, bp, float(g["U"]), float(g["dtau"]), Lx, Lx)
    for s in g["seeds"]:
        eng.add_chain(m, L, stab, int(s))
    eng.prepare(1)
    ok = [[True, True] for _ in g["seeds"]]   # still on trajectory (1 thread, 4 threads)
    for s in range(sweeps):
        eng.sweep(1)
        for c in range(len(g["seeds"])):
            f = eng.field(c)
            for v, key in enumerate(("fields", "fields_t4")):
                ok[c][v] = ok[c][v] and bool(np.array_equal(f, g[key][c][s]))
            assert any(ok[c]), f"chain {c} sweep {s}: off both reference trajectories"
    for c in range(len(g["seeds"])):
        cnt = eng.counters(c)
        if ok[c][0]:
            assert (cnt["attempts"], cnt["accepted"]) == tuple(int(x) for x in g["counters"][c])
        assert cnt["scratch_drift_samples"] == int(g["drift"][c][0])
        assert cnt["scratch_drift_max"] < 10 * max(g["drift"][c][1], 1e-4)
    eng.close()


def test_alternating_batched_with_forward_chains_equal():
    """An alternating engine's first (forward) sweep equals a forward engine's;
    after a backward sweep the two orders differ (slices visited in reverse)."""
    T, bp = dq.square_lattice(6, 6)
    engs = []
    for order in (dq.SWEEP_FORWARD, dq.SWEEP_ALTERNATING):
        e = dq.Engine(sweep_order=order)
        m = e.add_model(T, bp, 4.0, 0.1, 6, 6)
        for s in (3, 4, 5):
            e.add_chain(m, 20, 8, s)
        e.prepare(1)
        engs.append(e)
    for e in engs:
        e.sweep(1)
    for c in range(3):
        np.testing.assert_array_equal(engs[0].field(c), engs[1].field(c))
    for e in engs:
        e.close()
