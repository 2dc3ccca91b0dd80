"""Mixed-precision path vs the FP64 path, in lock step.

precision=mixed runs the wrap (green.c:509-548) and the delayed-update
flush (green.c:462-475) as FP64-emulated int8 split products on the tcgen05
tensor cores (8 balanced base-256 digits per line).  Stated bound, the one
the reference's own drift diagnostic (dqmc.c:64-98) is compared against:
max|G_mixed - G_FP64| <= 1e-8 at EVERY stabilization point, measured on the
wrapped G just before the rebuild replaces it (after the rebuild both are
the same FP64 function of the field, so a post-rebuild comparison would be
vacuous).  The two engines run from the same seeds; their accept/reject
decisions must be identical (bit-exact fields, counters, RNG), which makes
the snapshots comparable one to one.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")


def make(precision, Lx, U, L, stab, seeds, delay_rank=0, nbin=2, glog=0, order=0):
    T, bp = dq.square_lattice(Lx, Lx)
    eng = dq.Engine(precision=precision, delay_rank=delay_rank, green_log=glog,
                    sweep_order=order)
    m = eng.add_model(T, bp, U, 0.1, Lx, Lx, szz="af", sperp="af")
    for s in seeds:
        eng.add_chain(m, L, stab, s)
    eng.prepare(nbin)
    return eng


@pytest.mark.parametrize("Lx,L,stab", [(4, 10, 5), (6, 20, 8), (8, 40, 10), (12, 20, 10),
                                       (16, 80, 8), (24, 20, 5)])
def test_mixed_wrap_matches_fp64(Lx, L, stab):
    """One wrap of the same G: the split product is FP64-accurate (62-bit
    lines), so the two agree to about 1e-13 of |G|; lattices cover partial
    128-line tiles (16, 36, 64, 144 sites) and n = 576 (4.5 tiles)."""
    e64 = make(dq.PREC_FP64, Lx, 4.0, L, stab, [7])
    emx = make(dq.PREC_MIXED, Lx, 4.0, L, stab, [7])
    G0 = e64.green(0)
    np.testing.assert_array_equal(G0, emx.green(0))   # G from scratch is FP64 in both
    for l in (0, 1, L - 1):
        a, b = e64.wrap(0, l, G0), emx.wrap(0, l, G0)
        err = np.max(np.abs(a - b)) / np.max(np.abs(a))
        assert err <= 1e-11, (l, err)
    e64.close()
    emx.close()


def lockstep(Lx, U, L, stab, seeds, sweeps, delay_rank=0, order=0):
    M = -(-L // stab)
    per = M if order == 0 else M   # snapshots per sweep (one per stabilization point)
    cap = per * sweeps + 2
    e64 = make(dq.PREC_FP64, Lx, U, L, stab, seeds, delay_rank, glog=cap, order=order)
    emx = make(dq.PREC_MIXED, Lx, U, L, stab, seeds, delay_rank, glog=cap, order=order)
    for b in range(2):
        e64.sweep_measure(sweeps // 2, b)
        emx.sweep_measure(sweeps // 2, b)
    worst = 0.0
    for c in range(len(seeds)):
        np.testing.assert_array_equal(e64.field(c), emx.field(c))
        c64, cmx = e64.counters(c), emx.counters(c)
        for k in ("attempts", "accepted", "sweeps", "status"):
            assert c64[k] == cmx[k], k
        np.testing.assert_array_equal(c64["rng"], cmx["rng"])
        assert cmx["status"] == 0
        g64, gmx = e64.green_log(c), emx.green_log(c)
        assert len(g64) == len(gmx) and len(g64) >= sweeps * (M - 1)
        dG = np.max(np.abs(g64 - gmx), axis=(1, 2))
        worst = max(worst, float(dG.max()))
        s64, z64, p64 = e64.bins(c)
        smx, zmx, pmx = emx.bins(c)
        np.testing.assert_allclose(smx, s64, rtol=1e-7, atol=1e-9)
        np.testing.assert_allclose(zmx, z64, rtol=1e-7, atol=1e-9)
    e64.close()
    emx.close()
    return worst


@pytest.mark.parametrize("Lx,U,L,stab,sweeps,k", [(8, 4.0, 40, 10, 4, 16),
                                                  (16, 4.0, 80, 8, 2, 32)])
def test_mixed_lockstep_pre_rebuild(Lx, U, L, stab, sweeps, k):
    """8x8 beta=4 (the C2 lattice) and 16x16 beta=8 (the benchmark
    lattice): max|G_mixed - G_FP64| <= 1e-8 before every rebuild."""
    worst = lockstep(Lx, U, L, stab, [11, 12, 13], sweeps, delay_rank=k)
    assert worst <= 1e-8, worst


def test_mixed_lockstep_alternating():
    """Backward sweeps wrap with B^-1 G B (green.c:529-548), also split."""
    worst = lockstep(8, 4.0, 40, 10, [5, 6], 4, delay_rank=16, order=dq.SWEEP_ALTERNATING)
    assert worst <= 1e-8, worst


def test_fp64_green_log_is_the_wrapped_g():
    """The snapshot is G as wrapped: its distance to the rebuilt G is the
    engine's own drift (max over the snapshots = drift_max)."""
    e = make(dq.PREC_FP64, 6, 4.0, 20, 5, [3], glog=16)
    e.sweep(1)
    snaps = e.green_log(0)
    assert len(snaps) == 4
    c = e.counters(0)
    assert c["drift_samples"] == 4
    assert np.all(np.isfinite(snaps))
    e.close()
