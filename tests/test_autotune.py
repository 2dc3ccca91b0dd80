"""The autotuner's choice rule and cache (dqmc_b200/autotune.py), with a
fake trial in place of GPU timing."""
import pytest

from dqmc_b200 import autotune


def classes():
    return [dict(Lx=4, Ly=4, n=16, L=40, U=4.0, dtau=0.1, stab=8),
            dict(Lx=12, Ly=12, n=144, L=100, U=6.0, dtau=0.1, stab=8)]


def fake_trial(log):
    def trial(cls, k, pairs, stab):
        log.append((k, pairs, stab))
        out = []
        for c in cls:
            st = stab or c["stab"]   # 0: the class's own interval
            # larger intervals are faster; above 10 the drift of the big
            # class explodes; k = 32 paired is the fastest update
            cyc = c["n"] ** 3 * c["L"] / st * {(32, 2): 1.0, (32, 0): 1.03}.get((k, pairs), 1.2)
            drift = 1e-9 if (c["n"] < 100 or st <= 10) else 1e-2
            out.append((cyc, drift))
        return out
    return trial


def test_choose_prefers_fastest_within_the_default_interval_drift(tmp_path):
    log = []
    t = autotune.Tuner(cache_path=str(tmp_path / "c.json"), trial=fake_trial(log),
                       device_name="fake")
    small, big = t.tune(classes(), tune_stab=True)
    assert (small["delay_rank"], small["flush_pairs"], small["stab"]) == (32, 2, 16)
    # the big class may not go above 10: its drift there exceeds the
    # drift of the default interval 8
    assert (big["delay_rank"], big["flush_pairs"], big["stab"]) == (32, 2, 10)
    assert t.trials == len(autotune.DELAYS) * len(autotune.STABS)
    assert not small["cached"]


def test_cache_is_reused_per_device(tmp_path):
    log = []
    path = str(tmp_path / "c.json")
    autotune.Tuner(cache_path=path, trial=fake_trial(log), device_name="fake").tune(
        classes(), tune_stab=False)
    n0 = len(log)
    assert n0 == len(autotune.DELAYS)
    again = autotune.Tuner(cache_path=path, trial=fake_trial(log), device_name="fake")
    res = again.tune(classes(), tune_stab=False)
    assert len(log) == n0 and all(r["cached"] for r in res)
    assert all(r["stab"] == 8 for r in res)     # the interval stays fixed
    other = autotune.Tuner(cache_path=path, trial=fake_trial(log), device_name="other")
    other.tune(classes(), tune_stab=False)
    assert len(log) == 2 * n0


def test_default_kept_within_the_noise_margin():
    res = {(32, 0, 8): (100.0, 1e-9), (16, 2, 8): (97.0, 1e-9), (64, 2, 8): (94.0, 1e-9)}
    assert autotune.choose(res, 1e-6, (32, 0, 8)) == (64, 2, 8)
    res[(64, 2, 8)] = (96.0, 1e-9)
    assert autotune.choose(res, 1e-6, (32, 0, 8)) == (32, 0, 8)


def test_choose_falls_back_when_nothing_meets_the_tolerance():
    res = {(16, 1, 8): (5.0, 1.0), (32, 2, 8): (4.0, 2.0)}
    # the default interval's own drift is the limit: 1.0
    assert autotune.choose(res, 1e-6) == (16, 1, 8)
