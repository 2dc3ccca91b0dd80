"""The two batched workloads against the reference, chain by chain.

* Uneven batch: 64 chains of 4x4..12x12 (n = 16..144) with U drawn from
  {2,4,6} and beta from {1,...,10} (L = 10..100), seeds 1..64
  (dqmc_b200.workloads.uneven_batch), all in ONE engine / one launch per
  sweep.  Each chain is what the reference program runs with
  beta_list=<beta> seed=<seed> (beta index 0 keeps the seed,
  src/replica.c:17-34); golden vectors of eight chains covering every
  lattice size come from the reference run on its own
  (tests/golden/make_golden.py): field flips, counters and RNG bit-exact,
  G within the stabilization tolerance.
* Low-temperature lattice: 24x24 (n = 576), U = 8, dtau = 0.05, beta = 10
  (L = 200), stabilization every 5 slices, delay rank 64 (32-site blocks
  with paired rank <= 64 updates): two sweeps of a shortened L = 40 against
  the reference; at the full L = 200 the reference's own G is off by O(1)
  (particle-hole identity violated by 0.76), so there the engine is checked
  against that identity on its own two-spin path, and the mixed-precision
  path against the FP64 path in lock step.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")
from dqmc_b200.workloads import LOWT, uneven_batch  # noqa: E402


def g_close(G, g, c, tol=1e-8):
    """G against a golden summary: the full G (n <= 64), else its 32 x 32
    corner, every 7th row/column and its Frobenius norm."""
    scale = max(1.0, float(np.max(np.abs(G))))
    if f"G_{c}" in g.files:
        assert np.max(np.abs(G - g[f"G_{c}"])) <= tol * scale
        return
    assert np.max(np.abs(G[:32, :32] - g[f"G_corner_{c}"])) <= tol * scale
    assert np.max(np.abs(G[::7, ::7] - g[f"G_sub_{c}"])) <= tol * scale
    assert abs(np.linalg.norm(G) - float(g[f"G_fro_{c}"])) <= tol * scale * G.shape[0]


def batch_engine(precision=0, stab=8, delay_rank=0, glog=0):
    chains = uneven_batch()
    eng = dq.Engine(precision=precision, delay_rank=delay_rank, green_log=glog)
    models = {}
    for w in chains:
        key = (w["Lx"], w["U"])
        if key not in models:
            T, bp = dq.square_lattice(w["Lx"], w["Lx"])
            models[key] = eng.add_model(T, bp, w["U"], w["dtau"], w["Lx"], w["Lx"])
        eng.add_chain(models[key], w["L"], stab, w["seed"])
    eng.prepare(1)
    return eng, chains


def test_uneven_batch_matches_reference_chain_by_chain():
    g = golden("batch64_sel")
    sel = [int(c) for c in g["selection"]]
    eng, chains = batch_engine(stab=int(g["stab"]))
    assert len(chains) == 64
    for c in sel:
        np.testing.assert_array_equal(eng.field(c).ravel(), g[f"field0_{c}"].ravel())
    # chain 24 (12x12, U=6, beta=10) meets an acceptance decision at the
    # rounding level in its second sweep: the reference with one BLAS thread
    # and the same reference with four take it opposite ways, and either
    # trajectory is the reference's (both stored by make_golden.py)
    follows = {c: {"t1", "t4"} for c in sel}
    for s in range(int(g["sweeps"])):
        eng.sweep(1)
        for c in sel:
            f = eng.field(c).ravel()
            if not np.array_equal(f, g[f"fields_{c}"][s].ravel()):
                follows[c].discard("t1")
            if not np.array_equal(f, g[f"fields_t4_{c}"][s].ravel()):
                follows[c].discard("t4")
            assert follows[c], (c, s)
    for c in sel:
        if "t1" not in follows[c]:
            continue   # counters and G below belong to the one-thread trajectory
        cnt = eng.counters(c)
        ref = g[f"counters_{c}"][-1]
        assert (cnt["attempts"], cnt["accepted"], cnt["sweeps"], cnt["status"]) == tuple(ref)
        np.testing.assert_array_equal(cnt["rng"], g[f"rng_{c}"])
        g_close(eng.green(c), g, c)
    assert all(eng.counters(c)["status"] == 0 for c in range(64))
    eng.close()


def test_uneven_batch_mixed_precision_in_lock_step():
    """The batch in precision=mixed: the same flips as FP64 and
    max|G_mixed - G_FP64| <= 1e-8 before every rebuild, on every chain."""
    e64, _ = batch_engine(glog=32)
    emx, _ = batch_engine(precision=dq.PREC_MIXED, glog=32)
    e64.sweep(1)
    emx.sweep(1)
    worst = 0.0
    for c in range(64):
        np.testing.assert_array_equal(e64.field(c), emx.field(c))
        a, b = e64.green_log(c), emx.green_log(c)
        assert len(a) == len(b) > 0
        worst = max(worst, float(np.max(np.abs(a - b))))
    assert worst <= 1e-8, worst
    e64.close()
    emx.close()


def lowt_chain(L, seed, precision=0, glog=0):
    w = LOWT
    eng = dq.Engine(precision=precision, delay_rank=w["delay_rank"], green_log=glog)
    T, bp = dq.square_lattice(w["Lx"], w["Lx"])
    m = eng.add_model(T, bp, w["U"], w["dtau"], w["Lx"], w["Lx"])
    eng.add_chain(m, L, w["stab"], seed)
    eng.prepare(1)
    return eng


def test_lowt_24x24_short_matches_reference():
    """L = 40 (beta = 2): fields, counters and RNG bit-exact over two sweeps,
    the initial G to 1e-6 of max|G|.  The reference's G is less accurate
    here than that: its two-spin path gives a G_down that misses the
    particle-hole map of its G_up by 1.9e-4 at the start (stored in the
    golden file) and by O(1) after a sweep, while this engine's two paths
    agree to 1e-12 (below)."""
    g = golden("sq24_lowt")
    tag = "short"
    Lx, L, stab, seed, sweeps = (int(x) for x in g[f"{tag}_params"])
    assert (Lx, stab) == (LOWT["Lx"], LOWT["stab"])
    eng = lowt_chain(L, seed)
    np.testing.assert_array_equal(eng.field(0).ravel(), g[f"{tag}_field0"].ravel())
    G0 = eng.green(0)
    scale = max(1.0, float(np.max(np.abs(G0))))
    assert np.max(np.abs(G0[:32, :32] - g[f"{tag}_G_corner0"])) <= 1e-6 * scale
    for s in range(sweeps):
        eng.sweep(1)
        np.testing.assert_array_equal(eng.field(0).ravel(), g[f"{tag}_fields"][s].ravel())
    cnt = eng.counters(0)
    assert (cnt["attempts"], cnt["accepted"], cnt["sweeps"], cnt["status"]) == \
        tuple(g[f"{tag}_counters"][-1])
    np.testing.assert_array_equal(cnt["rng"], g[f"{tag}_rng"])
    # G after the sweeps is not compared: on this lattice the reference's own
    # two-spin G_down misses the particle-hole map of its G_up by 7.7 after
    # one sweep and 0.52 after two (0.00019 at the start), so its G is no
    # yardstick here; the engine's accuracy is checked below by the same
    # identity on its own two-spin path
    assert np.all(np.isfinite(eng.green(0)))
    eng.close()


@pytest.mark.parametrize("L,seed,bound", [(40, 102, 1e-11), (200, 101, 1e-9)])
def test_lowt_24x24_particle_hole_consistency(L, seed, bound):
    """At beta = 10 (L = 200) the reference's G from scratch is no longer a
    usable reference: its G_down misses the particle-hole map
    I - P G_up^T P of its G_up by 0.76 (0.00019 at L = 40; the golden file
    stores both).  This engine builds G_up and G_down independently on its
    two-spin path (separate sigma = +1 / -1 factors and UDV stacks, columns
    pre-pivoted by norm); they satisfy the identity to the bound, at the
    start and after a sweep, and the field stream matches the reference."""
    g = golden("sq24_lowt")
    tag = "full" if L == 200 else "short"
    assert float(g[f"{tag}_ref_ph_violation0"]) > 1e3 * bound
    w = LOWT
    T, bp = dq.square_lattice(w["Lx"], w["Lx"])
    P = np.diag(bp.astype(float))
    eng = dq.Engine(delay_rank=32)   # the two-spin path takes k <= 32
    m = eng.add_model(T, bp, w["U"], w["dtau"], w["Lx"], w["Lx"], two_spin=True)
    eng.add_chain(m, L, w["stab"], seed)
    eng.prepare(1)
    np.testing.assert_array_equal(eng.field(0).ravel(), g[f"{tag}_field0"].ravel())
    n = w["Lx"] ** 2
    for _ in range(2):
        Gu, Gd = eng.green(0), eng.green_down(0)
        assert np.max(np.abs(Gd - (np.eye(n) - P @ Gu.T @ P))) <= bound
        eng.sweep(1)
    assert eng.counters(0)["status"] == 0
    eng.close()


@pytest.mark.parametrize("L,seed", [(40, 102), (200, 101)])
def test_lowt_24x24_mixed_precision_in_lock_step(L, seed):
    M = L // LOWT["stab"]
    e64 = lowt_chain(L, seed, glog=M + 2)
    emx = lowt_chain(L, seed, precision=dq.PREC_MIXED, glog=M + 2)
    e64.sweep(1)
    emx.sweep(1)
    np.testing.assert_array_equal(e64.field(0), emx.field(0))
    a, b = e64.green_log(0), emx.green_log(0)
    assert len(a) == len(b) == M
    worst = float(np.max(np.abs(a - b)))
    assert worst <= 1e-8, worst
    e64.close()
    emx.close()
