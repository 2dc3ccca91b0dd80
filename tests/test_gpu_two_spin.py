"""The two-spin path (the reference's use_ph = 0, src/dqmc.c:641-813) on the
GPU against the reference (golden vectors made by the reference itself,
tests/golden/make_golden.py --only-two-spin).

Cases: the PH point forced onto the two-spin path (the reference's
ph_symmetric = 0 override, tests/test_dqmc_stack.c:81), a non-bipartite
3-site ring at half filling, and a doped 4x4 lattice (mu = 0.7).  Bars as
for the PH path: field flips, counters, running sign and RNG state
bit-exact, G_up and G_down within 1e-9, the measured energies within 1e-9.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")

CASES = ["sq4_2spin", "chain3_2spin", "sq4_mu"]


def engine_for(g, nbin=1, delay_rank=0):
    kind, Lx, Ly, L, stab, seed, sweeps, half, force = (int(x) for x in g["params"])
    if kind == 0:
        T, bp = dq.chain_lattice(Lx)
        Ly = 1
        if Lx % 2:
            bp = None   # odd ring: not bipartite
    else:
        T, bp = dq.square_lattice(Lx, Ly)
    eng = dq.Engine(delay_rank=delay_rank)
    m = eng.add_model(T, bp, float(g["U"]), float(g["dtau"]), Lx, Ly,
                      mu=None if half else float(g["mu"]), two_spin=bool(force))
    eng.add_chain(m, L, stab, seed)
    eng.prepare(nbin)
    return eng, sweeps


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("kb", [0, 1, 5])
def test_two_spin_matches_reference(name, kb):
    """kb: site-block size (0 = by n; 1 and 5 give several blocks, each
    flushing both spins)."""
    g = golden(name)
    eng, sweeps = engine_for(g, nbin=int(g["params"][6]), delay_rank=kb)
    np.testing.assert_array_equal(eng.field(0), g["field0"])
    assert np.max(np.abs(eng.green(0) - g["Gu0"])) < 1e-10
    assert np.max(np.abs(eng.green_down(0) - g["Gd0"])) < 1e-10
    assert eng.counters(0)["sign"] == float(g["sign0"])
    for s in range(sweeps):
        eng.sweep_measure(1, s)
        np.testing.assert_array_equal(eng.field(0), g["fields"][s])
        c = eng.counters(0)
        att, acc, sw, status = (int(x) for x in g["counters"][s])
        assert (c["attempts"], c["accepted"], c["sweeps"], c["status"]) == (att, acc, sw, status)
        assert c["sign"] == float(g["sign"][s])
        assert np.max(np.abs(eng.green(0) - g["Gu"][s])) < 1e-9, s
        assert np.max(np.abs(eng.green_down(0) - g["Gd"][s])) < 1e-9, s
    np.testing.assert_array_equal(eng.counters(0)["rng"], g["rng_end"])
    sc, _, _ = eng.bins(0)
    for s in range(sweeps):
        E, ekin, eint, ntot, dbl = g["meas"][s]
        sign = float(g["sign"][s])
        assert abs(sc[s, 0] - sign * E) < 1e-9
        assert abs(sc[s, 3] - sign * ntot) < 1e-9
        assert abs(sc[s, 4] - sign * dbl) < 1e-9
        assert sc[s, 5] == sign
    eng.close()


def test_forced_two_spin_equals_ph_path():
    """At half filling on a bipartite lattice both paths take the same
    decisions, and the evolved G_down equals the PH map of G_up
    (tests/test_dqmc_stack.c:68-118)."""
    T, bp = dq.square_lattice(6, 6)
    out = []
    for two in (False, True):
        e = dq.Engine()
        m = e.add_model(T, bp, 4.0, 0.1, 6, 6, two_spin=two)
        e.add_chain(m, 30, 7, 13)
        e.prepare(1)
        e.sweep(3)
        out.append((e.field(0), e.green(0), e.green_down(0), e.counters(0)))
        e.close()
    (f0, gu0, gd0, c0), (f1, gu1, gd1, c1) = out
    np.testing.assert_array_equal(f0, f1)
    assert (c0["attempts"], c0["accepted"]) == (c1["attempts"], c1["accepted"])
    assert np.max(np.abs(gu0 - gu1)) < 1e-9 and np.max(np.abs(gd0 - gd1)) < 1e-9
    assert c1["sign"] == 1.0 and c1["status"] == 0


def test_two_spin_rejects_alternating_and_mixed():
    T, bp = dq.square_lattice(4, 4)
    for kw in (dict(sweep_order=dq.SWEEP_ALTERNATING), dict(precision=dq.PREC_MIXED)):
        e = dq.Engine(**kw)
        m = e.add_model(T, bp, 4.0, 0.1, 4, 4, mu=0.5)
        e.add_chain(m, 10, 5, 1)
        with pytest.raises(dq.DqmcError):
            e.prepare(1)
        e.close()
