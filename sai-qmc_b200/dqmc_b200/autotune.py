"""Autotuner for batched chains: delay rank, flush grouping and (where the
input leaves it free) the stabilization interval, per size class.

A size class is (n, L, U, dtau, particle-hole path).  The tuner times every
candidate setting on ALL classes of a batch at once: one engine per
candidate holds one chain of each class (one CTA, one SM each), and each
chain's own device cycle counters (dqmc_read_profile) give that class's
sweep time, so a candidate costs one trial launch, not one per class.  Two
sweeps are timed after a first one that builds the B-block cache.

Choosing: the fastest candidate of a class whose stabilization drift
max|G_wrapped - G_rebuilt| stays at or below max(drift_tol, the drift of
the reference's default interval 8), so a tuned interval never costs
accuracy against the reference's default; and the engine's default setting
(k = 32, automatic pairing, interval 8) stays unless a candidate is at
least 5% faster, a margin above the noise of a two-sweep trial.  The
delay rank and the flush grouping do not change the accept/reject
sequence; the interval changes it only at the rounding level.  Results are cached per device name in a JSON
file ($DQMC_TUNE_CACHE, default ~/.cache/dqmc_b200/tune.json).
"""
from __future__ import annotations

import json
import os

# (k, DQMC_PAIRS_*): the engine's default (32, AUTO) first
DELAYS = ((32, 0), (16, 1), (16, 2), (32, 1), (32, 2), (48, 2), (64, 2))
STABS = (5, 8, 10, 12, 16)
DEFAULT_STAB = 8
MARGIN = 0.05        # leave the default only for a gain above trial noise
TRIAL_SWEEPS = 2


def class_key(device_name, c, tune_stab):
    return (f"{device_name}|n={c['n']}|L={c['L']}|U={c['U']:g}|dtau={c['dtau']:g}|"
            f"ph={int(c.get('ph', True))}|stab={'free' if tune_stab else c['stab']}")


def choose(results, drift_tol, default=None):
    """results: {(k, pairs, stab): (cycles, drift)} of one class -> the
    chosen (k, pairs, stab): the fastest whose drift is within the limit,
    unless it beats the default setting by less than MARGIN."""
    ref = [d for (k, p, s), (_, d) in results.items() if s == DEFAULT_STAB]
    limit = max(drift_tol, min(ref)) if ref else drift_tol
    ok = {key: v for key, v in results.items() if v[1] <= limit and v[1] == v[1]}
    pool = ok or results
    best = min(pool, key=lambda key: (pool[key][0], key))
    if default in pool and pool[best][0] > (1.0 - MARGIN) * pool[default][0]:
        return default
    return best


class Tuner:
    def __init__(self, device=0, cache_path=None, drift_tol=1e-6, trial=None, device_name=None):
        self.device = device
        self.cache_path = cache_path or os.environ.get("DQMC_TUNE_CACHE") or os.path.join(
            os.path.expanduser("~"), ".cache", "dqmc_b200", "tune.json")
        self.drift_tol = drift_tol
        self._trial = trial or self._engine_trial
        self.device_name = device_name
        self.trials = 0

    # ------------------------------------------------------------ cache
    def _load(self):
        try:
            with open(self.cache_path) as f:
                return json.load(f)
        except (OSError, ValueError):
            return {}

    def _save(self, cache):
        os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def _name(self):
        if self.device_name is None:
            import torch
            self.device_name = torch.cuda.get_device_name(self.device)
        return self.device_name

    # ------------------------------------------------------------ trials
    def _engine_trial(self, classes, k, pairs, stab):
        """One engine, one chain per class with this setting; returns
        [(cycles per sweep, drift)] per class."""
        from . import Engine, square_lattice
        eng = Engine(device=self.device, delay_rank=k, flush_pairs=pairs)
        models = {}
        for c in classes:
            key = (c["Lx"], c["Ly"], c["U"], c["dtau"])
            if key not in models:
                T, bp = square_lattice(c["Lx"], c["Ly"])
                models[key] = eng.add_model(T, bp, c["U"], c["dtau"], c["Lx"], c["Ly"])
            eng.add_chain(models[key], c["L"], stab if stab else c["stab"], c.get("seed", 1))
        eng.prepare(1)
        eng.sweep(1)
        p0 = [sum(eng.profile(i).values()) for i in range(len(classes))]
        eng.sweep(TRIAL_SWEEPS)
        eng.sync()
        out = []
        for i in range(len(classes)):
            cyc = (sum(eng.profile(i).values()) - p0[i]) / TRIAL_SWEEPS
            cnt = eng.counters(i)
            out.append((float(cyc), float(cnt["drift_max"]) if cnt["status"] == 0
                        else float("inf")))
        eng.close()
        return out

    def tune(self, classes, tune_stab):
        """classes: dicts with Lx, Ly, n, L, U, dtau, stab (used when the
        interval is not tuned) and optionally seed.  Returns one dict per
        class: delay_rank, flush_pairs, stab, cycles, drift, cached."""
        name = self._name()
        cache = self._load()
        keys = [class_key(name, c, tune_stab) for c in classes]
        todo = [i for i, k in enumerate(keys) if k not in cache]
        if todo:
            sub = [classes[i] for i in todo]
            stabs = STABS if tune_stab else (0,)
            results = [dict() for _ in sub]
            for k, pairs in DELAYS:
                for s in stabs:
                    self.trials += 1
                    for j, r in enumerate(self._trial(sub, k, pairs, s)):
                        results[j][(k, pairs, s if s else sub[j]["stab"])] = r
            for j, i in enumerate(todo):
                dflt = (DELAYS[0][0], DELAYS[0][1], DEFAULT_STAB if tune_stab else sub[j]["stab"])
                k, pairs, s = choose(results[j], self.drift_tol, dflt)
                cyc, dr = results[j][(k, pairs, s)]
                cache[keys[i]] = {"delay_rank": k, "flush_pairs": pairs, "stab": s,
                                  "cycles": cyc, "drift": dr}
            self._save(cache)
        return [dict(cache[k], cached=(i not in todo)) for i, k in enumerate(keys)]
