"""One chain advanced by a thread-block cluster (dqmc_engine_desc.chain_ctas).

Rank 0 of the cluster runs the sweep; every rank forms its share of the
output tiles of the wrap, the B-block products and the delayed-update G
update.  Each output element is formed by the same DMMA instruction
sequence whatever the tile shape and share, so the bar is equality with
the one-CTA engine: field flips, counters, RNG state and bins bit-exact,
G equal to the last bit.  One case is also held against the reference's
own golden vectors (flips and RNG bit-exact, G within 1e-9).
"""
import numpy as np
import pytest

from conftest import case_args, golden

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")


def build(lats, L, stab, seeds, ctas, U=4.0, dtau=0.1, nbin=1, **kw):
    eng = dq.Engine(chain_ctas=ctas, **kw)
    for (Lx, Ly, mu), seed in zip(lats, seeds):
        T, bp = dq.square_lattice(Lx, Ly)
        m = eng.add_model(T, bp, U, dtau, Lx, Ly, szz="all", sperp="all", mu=mu)
        eng.add_chain(m, L, stab, seed)
    eng.prepare(nbin)
    return eng


def run_pair(lats, L, stab, seeds, ctas, sweeps=2, **kw):
    one = build(lats, L, stab, seeds, 1, nbin=sweeps, **kw)
    cl = build(lats, L, stab, seeds, ctas, nbin=sweeps, **kw)
    for s in range(sweeps):
        one.sweep_measure(1, s)
        cl.sweep_measure(1, s)
    one.sync()
    cl.sync()
    for c in range(len(seeds)):
        np.testing.assert_array_equal(cl.field(c), one.field(c))
        a, b = cl.counters(c), one.counters(c)
        assert a["status"] == 0 and b["status"] == 0
        for k in ("attempts", "accepted", "sweeps", "sign", "drift_max"):
            assert a[k] == b[k], (c, k, a[k], b[k])
        np.testing.assert_array_equal(a["rng"], b["rng"])
        assert np.array_equal(cl.green(c), one.green(c)), \
            float(np.max(np.abs(cl.green(c) - one.green(c))))
        for x, y in zip(cl.bins(c), one.bins(c)):
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))
    one.close()
    cl.close()


@pytest.mark.parametrize("ctas", [2, 3, 4, 8])
def test_cluster_equals_one_cta_8x8(ctas):
    run_pair([(8, 8, None)], 40, 10, [7], ctas)


@pytest.mark.parametrize("ctas", [4, 8, 12, 16])
def test_cluster_equals_one_cta_16x16(ctas):
    """n = 256: 128x128 or 64x64 tiles by share, paired site blocks."""
    run_pair([(16, 16, None)], 16, 8, [11], ctas)


def test_cluster_uneven_batch_and_small_tiles():
    """Chains of n = 16 (SIMT tiles), 64, 100 and 144 in one launch of
    four-CTA clusters, chains ordered by cost."""
    run_pair([(4, 4, None), (8, 8, None), (10, 10, None), (12, 12, None)], 20, 5,
             [1, 2, 3, 4], 4)


def test_cluster_alternating_order():
    """Backward sweeps: B^-1 G B wraps and the prefix stack's B-blocks."""
    run_pair([(10, 10, None)], 24, 6, [5], 4, sweeps=4,
             sweep_order=dq.SWEEP_ALTERNATING)


def test_cluster_two_spin_path():
    """G_up and G_down evolved separately (doped), both G updates split."""
    run_pair([(6, 6, 0.7)], 20, 5, [9], 2)


def test_cluster_with_reference_drift_rebuild():
    """The reference-definition rebuild from scratch between stabilizations
    (its B-block chain runs as split commands too)."""
    run_pair([(8, 8, None)], 20, 5, [3], 4, drift=dq.DRIFT_STAB | dq.DRIFT_SCRATCH)


def test_cluster_matches_reference_golden():
    g = golden("sq8_b4")
    a = case_args(g)
    T, bp = dq.square_lattice(a["Lx"], a["Ly"])
    eng = dq.Engine(chain_ctas=4)
    m = eng.add_model(T, bp, a["U"], a["dtau"], a["Lx"], a["Ly"], szz=a["selector"],
                      sperp=a["selector"])
    eng.add_chain(m, a["L"], a["stab"], a["seed"])
    eng.prepare(a["sweeps"])
    for s in range(a["sweeps"]):
        eng.sweep_measure(1, s)
        np.testing.assert_array_equal(eng.field(0), g["fields"][s])
        att, acc, sw, status = (int(x) for x in g["counters"][s])
        c = eng.counters(0)
        assert (c["attempts"], c["accepted"], c["sweeps"], c["status"]) == \
            (att, acc, sw, status)
        assert np.max(np.abs(eng.green(0) - g["Gs"][s])) < 1e-9
    np.testing.assert_array_equal(eng.counters(0)["rng"], g["rng_end"])
    eng.close()


@pytest.mark.parametrize("ctas", [4, 16])
def test_cluster_mixed_precision_equals_one_cta(ctas):
    """Split products (tcgen05 kind::i8) shared over the cluster: each rank
    splits a range of lines and forms a share of the tiles on its own tensor
    memory; the same digits and tiles as one CTA."""
    run_pair([(16, 16, None)], 16, 8, [11], ctas, precision=dq.PREC_MIXED)


def test_cluster_mixed_precision_alternating_uneven():
    run_pair([(8, 8, None), (12, 12, None)], 20, 5, [3, 4], 4, sweeps=4,
             precision=dq.PREC_MIXED, sweep_order=dq.SWEEP_ALTERNATING)


def test_cluster_rejects_bad_settings():
    with pytest.raises(dq.DqmcError, match="chain_ctas"):
        dq.Engine(chain_ctas=17)
    with pytest.raises(dq.DqmcError, match="one CTA per SM"):
        dq.Engine(chain_ctas=4, ctas_per_sm=2)


def test_cluster_size_chosen_automatically():
    """chain_ctas = 0: a cluster per chain for batches of fewer chains than
    SMs with n >= 128, one CTA per chain otherwise."""
    def residency(Lx, nch, **kw):
        T, bp = dq.square_lattice(Lx, Lx)
        e = dq.Engine(**kw)
        m = e.add_model(T, bp, 4.0, 0.1, Lx, Lx)
        for c in range(nch):
            e.add_chain(m, 8, 8, c + 1)
        e.prepare(1)
        r = e.residency()
        e.close()
        return r
    per_sm, cc, ncoop = residency(16, 1)
    assert per_sm == 1 and cc > 1 and ncoop == 1
    assert residency(16, 1, chain_ctas=1)[:2] == (1, 1)
    assert residency(16, 1, precision=dq.PREC_MIXED)[1] == cc
    assert residency(8, 1)[:2] == (1, 1)
    per_sm, cc8, ncoop8 = residency(16, 8)
    assert per_sm == 1 and 1 < cc8 <= cc and ncoop8 == 8


def test_cluster_and_packed_chains_in_one_launch():
    """cluster_chains: the two most expensive of six uneven chains on a
    four-CTA cluster each, the other four packed one per CTA in the same
    launch; everything equal to one CTA per chain."""
    lats = [(4, 4, None), (6, 6, None), (8, 8, None), (10, 10, None), (12, 12, None),
            (16, 16, None)]
    run_pair(lats, 16, 8, [1, 2, 3, 4, 5, 6], 4, cluster_chains=2)
    e = build(lats, 16, 8, [1, 2, 3, 4, 5, 6], 4, cluster_chains=2)
    assert e.residency() == (1, 4, 2)
    e.close()


@pytest.mark.parametrize("prec", [dq.PREC_FP64, dq.PREC_MIXED])
def test_cluster_chain_failure_stops_only_that_chain(prec):
    """A chain on a cluster whose G is corrupted from the host stops at its
    first stabilization point (rank 0 leaves the sweep and releases the other
    ranks); its batch-mates, also on clusters, equal a clean run."""
    lats, seeds = [(16, 16, None)] * 3, [3, 4, 5]
    clean = build(lats, 16, 8, seeds, 4, precision=prec)
    hit = build(lats, 16, 8, seeds, 4, precision=prec)
    G = hit.green(1)
    G[2, 3] = np.nan
    hit.write_green(1, G)
    clean.sweep(2)
    hit.sweep(2)
    c = hit.counters(1)
    assert c["status"] & 1 and c["sign"] == 0.0 and c["sweeps"] == 0
    for k in (0, 2):
        np.testing.assert_array_equal(hit.field(k), clean.field(k))
        assert hit.counters(k)["status"] == 0
        assert np.array_equal(hit.green(k), clean.green(k))
    hit.sweep(1)                                   # the frozen chain stays frozen
    assert hit.counters(1)["attempts"] == c["attempts"]
    clean.close()
    hit.close()


@pytest.mark.parametrize("rebuild", [dq.REBUILD_TWO_SIDED, dq.REBUILD_CENTERED])
def test_cluster_two_sided_rebuild(rebuild):
    """G from the two boundary factors (its QR solve and triangular solves run
    as cluster commands) with UDV scale records on."""
    run_pair([(10, 10, None)], 24, 6, [5], 4, sweeps=3, green_rebuild=rebuild, udv_diag=1)
