"""green_rebuild=two_sided / centered on the GPU vs the reference.

The two-sided reconstruction forms G = (1 + L R)^-1 from the two boundary
factors without combining them (src/linalg.c:1117-1389).  Bars as for the
combine path: the reference's n=4 two-sided fixture (log D over 300 decades,
det sign -1) within 1e-9 relative with the same sign
(tests/test_udv_phase6a_fixture.c:136-158); sweeps with the reference's own
two-sided / centered rebuild (golden vectors from the reference) with
bit-exact flips, counters and RNG and G within 1e-9.
"""
import numpy as np
import pytest

from conftest import golden, rel_err

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")

CASES = ["sq4_b4_2s", "sq8_b4_2s", "chain4_ctr", "sq6_b2_2s_alt"]


def test_two_sided_fixture():
    g = golden("udv_two_sided_fixture")
    G, ds = dq.udv_green2(g["UL"], g["DL"], g["TL"], float(g["off_L"]),
                          g["UR"], g["DR"], g["TR"], float(g["off_R"]))
    assert ds == int(g["det_sign"])
    assert rel_err(G, g["G"]) <= 1e-9


@pytest.mark.parametrize("name", CASES)
def test_rebuild_modes_match_reference(name):
    g = golden(name)
    kind, Lx, Ly, L, stab, seed, sweeps, alt, rb = (int(x) for x in g["params"])
    if kind == 0:
        T, bp = dq.chain_lattice(Lx)
        Ly = 1
    else:
        T, bp = dq.square_lattice(Lx, Ly)
    eng = dq.Engine(sweep_order=dq.SWEEP_ALTERNATING if alt else dq.SWEEP_FORWARD,
                    green_rebuild=rb)
    m = eng.add_model(T, bp, float(g["U"]), float(g["dtau"]), Lx, Ly)
    eng.add_chain(m, L, stab, seed)
    eng.prepare(1)
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


def test_two_sided_equals_combine_on_same_field():
    """Both reconstructions give the same G for the same field (they differ
    only in rounding): one forward sweep each from the same seed."""
    T, bp = dq.square_lattice(8, 8)
    gs = []
    for rb in (dq.REBUILD_COMBINE, dq.REBUILD_TWO_SIDED):
        e = dq.Engine(green_rebuild=rb)
        m = e.add_model(T, bp, 4.0, 0.1, 8, 8)
        e.add_chain(m, 40, 10, 5)
        e.prepare(1)
        e.sweep(1)
        gs.append((e.field(0), e.green(0), e.counters(0)["drift_max"]))
        e.close()
    np.testing.assert_array_equal(gs[0][0], gs[1][0])
    assert np.max(np.abs(gs[0][1] - gs[1][1])) < 1e-9
    assert gs[1][2] < 1e-6
