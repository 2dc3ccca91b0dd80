"""The autotuner on the GPU: per-class settings for a batch of uneven
chains, applied per chain (dqmc_chain_tune), leave every trajectory equal
to the untuned batch's (the delay rank and flush grouping change only how
G is updated, not the accept/reject sequence)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

dq = pytest.importorskip("dqmc_b200")
from dqmc_b200 import autotune  # noqa: E402


def test_tuned_batch_follows_the_untuned_trajectories(tmp_path):
    specs = [(4, 2.0, 20), (6, 4.0, 20), (8, 4.0, 40), (10, 2.0, 20), (12, 4.0, 20)]
    classes = [dict(Lx=Lx, Ly=Lx, n=Lx * Lx, L=L, U=U, dtau=0.1, stab=8)
               for Lx, U, L in specs]
    t = autotune.Tuner(cache_path=str(tmp_path / "tune.json"))
    choice = t.tune(classes, tune_stab=False)
    assert t.trials == len(autotune.DELAYS)
    assert all(c["stab"] == 8 and np.isfinite(c["cycles"]) for c in choice)

    def batch(tuned):
        eng = dq.Engine()
        for i, (c, ch) in enumerate(zip(classes, choice)):
            T, bp = dq.square_lattice(c["Lx"], c["Ly"])
            m = eng.add_model(T, bp, c["U"], c["dtau"], c["Lx"], c["Ly"])
            for r in range(3):
                cid = eng.add_chain(m, c["L"], c["stab"], 100 * i + r + 1)
                if tuned:
                    eng.tune_chain(cid, ch["delay_rank"], ch["flush_pairs"])
        eng.prepare(1)
        eng.sweep(2)
        return eng

    a, b = batch(False), batch(True)
    for c in range(3 * len(classes)):
        np.testing.assert_array_equal(a.field(c), b.field(c))
        assert b.counters(c)["status"] == 0
        assert np.max(np.abs(a.green(c) - b.green(c))) < 1e-9
    a.close()
    b.close()
    again = autotune.Tuner(cache_path=str(tmp_path / "tune.json")).tune(classes, tune_stab=False)
    assert all(r["cached"] for r in again)
