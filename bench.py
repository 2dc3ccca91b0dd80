#!/usr/bin/env python3
"""Benchmark of the BSS determinant-QMC sweep on one B200 (or N, as replicas).

Workload (the lattice the headline metric is quoted on): 16x16 periodic
square lattice, t=-1, U=4, dtau=0.1, beta=8 (L=80), stabilization every 8
slices, delayed-update site blocks of 32, many independent replica chains
(seeds replica_seed(11, 0, r), src/replica.c:17-34) advancing together.
A step is one forward sweep of every chain followed by the fused
equal-time measurement.  value = whole-job field updates/s
(chains * n * L per step / device time, max over ranks).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--chains B]
  python bench.py --impl reference ...   # the reference CPU code, host cores

--gpus N > 1 without torchrun starts N ranks itself (one per GPU,
dqmc_b200.launch); under torchrun each rank runs as started.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "sai-qmc_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = ("field updates/s, 16x16 U=4 β=8: batched mixed vs plain FP64 GPU, "
          "max|ΔG|≤1e-8")
UNIT = "field updates/s"
LX, U, DTAU, BETA, STAB, KB, SEED = 16, 4.0, 0.1, 8.0, 8, 32, 11
N_SITES = LX * LX
L_SLICES = int(round(BETA / DTAU))
INT8_DENSE_OPS = 4.5e15   # nominal dense int8 tensor rate of a B200
SM_MAX_MHZ = 1965
L2_BYTES = 126 * 2**20


def workload_name(chains):
    return (f"16x16 square pbc, U=4, dtau=0.1, beta=8 (L=80), stab=8, delay rank 32, "
            f"{chains} replica chains per GPU, seeds replica_seed(11, 0, r)")


# --------------------------------------------------------------- helpers
def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def flops_per_chain_sweep(n, L, s, accepted):
    """Algorithmic floating-point work of one forward sweep of one chain,
    as the reference's algorithm spends it (PH path, combine rebuild;
    multiply-adds count 2 flops; M = ceil(L/s) blocks, a = accepted / (n L)):

      F = 4 n^3 L                        wrap: 2 GEMMs per slice
        + 2 a n^3 L                      rank-k flushes: 2 n^2 per accepted flip
        + (2M-1) [2 n^3 (s-1) + 6.7 n^3] B-block products and one QR-based
                                         lmul/rmul per block (stack and left)
        + (M-1) 19 n^3 + 10.3 n^3        combine + G from UDV per boundary

    This is the unit against which the roofline is reported (16x16, beta=8,
    stab=8: about 1.0e3 n^3 = 16.7 GFLOP per chain-sweep).  The engine
    executes less (B-blocks cached across sweeps, Q applied without being
    formed): see executed_flops_per_chain_sweep.
    """
    M = (L + s - 1) // s
    n3 = float(n) ** 3
    a = accepted / float(n * L)
    return (4 * n3 * L + 2 * a * n3 * L + (2 * M - 1) * (2 * n3 * (s - 1) + 6.7 * n3)
            + (M - 1) * 19 * n3 + 10.3 * n3)


def executed_flops_per_chain_sweep(n, L, s, accepted):
    """Floating-point work this engine performs per chain-sweep:
      wrap            2 GEMMs per slice                      4 n^3 L
      flush           rank-m updates of G                    2 n^2 * accepted
      B-block         (len-1) GEMMs per block, left pass     2 n^3 (L - M)
      suffix rmul     GEMM + QR + Q applied from the right   (4 + 4/3) n^3 (M-1)
      left lmul       GEMM + QR + form Q + triangular GEMM   (3 + 8/3) n^3 M
      combine         GEMM + QR + right-apply + triangular   (5 + 4/3) n^3 (M-1)
      G from UDV      QR + apply Q^T + triangular solve      (4/3 + 2 + 1) n^3 M
    """
    M = (L + s - 1) // s
    n3 = float(n) ** 3
    return (4 * n3 * L + 2.0 * n * n * accepted + 2 * n3 * (L - M)
            + (4 + 4 / 3) * n3 * (M - 1) + (3 + 8 / 3) * n3 * M
            + (5 + 4 / 3) * n3 * (M - 1) + (4 / 3 + 3) * n3 * M)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9 or parts[0] != str(self.idx):
                    continue
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        mhz = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(mhz) if mhz else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "power_w_max": max(float(r[3]) for r in rows
                                   if r[3].replace(".", "").isdigit()) if rows else None,
                "samples": len(rows), "reasons": reasons}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            return int(ids[local_rank])
    return local_rank


def fp64_gemm_peak_tflops():
    """cuBLAS DGEMM (torch.matmul, float64, 8192^3), best of 5: the measured
    FP64 tensor-core ceiling the sweep kernel's roofline is quoted against."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def traffic_per_chain_sweep(mixed=False):
    """DRAM bytes per chain-sweep of the sweep kernel from the committed ncu
    summary (profiles/), or None when no capture has been summarized."""
    path = os.path.join(ROOT, "profiles", "k_sweep_mixed_16x16_ncu.md" if mixed
                        else "k_sweep_16x16_ncu.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("dram_bytes_per_chain_sweep:"):
                return float(line.split(":", 1)[1])
    return None


# ------------------------------------------------------ reference CPU arm
def reference_cpu(steps, warmup, chains=None):
    """The reference's own sweep (dqmc_sweep, src/dqmc.c:952) on the host
    cores: one chain per core, each step one sweep of every chain, threads
    released from the GIL inside the C calls.  Falls back to the oracle
    restatement when the reference could not be compiled."""
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    from oracle.bind import LAT_SQUARE, Oracle, Reference
    cores = len(os.sched_getaffinity(0))
    chains = chains or cores
    if Reference.available():
        lib, kind = Reference(), "reference"
    else:
        lib, kind = Oracle(), "port"
    seeds = [lib.replica_seed(SEED, 0, r) for r in range(chains)]
    objs = [None] * chains

    def make(i):
        objs[i] = lib.chain(LAT_SQUARE, LX, LX, U, DTAU, L_SLICES, STAB, seeds[i])

    def parallel(fn):
        th = [threading.Thread(target=fn, args=(i,)) for i in range(chains)]
        for t in th:
            t.start()
        for t in th:
            t.join()

    parallel(make)
    for _ in range(warmup):
        parallel(lambda i: objs[i].sweep(1))
    t0 = time.perf_counter()
    for _ in range(steps):
        parallel(lambda i: objs[i].sweep(1))
    dt = time.perf_counter() - t0
    for o in objs:
        o.free()
    value = chains * N_SITES * L_SLICES * steps / dt
    sample = (f"{chains} chains x {steps} sweeps of the 16x16 U=4 beta=8 stab=8 workload, "
              f"one chain per host core, {dt:.1f} s wall")
    return {"value": value, "unit": UNIT, "cores": min(cores, chains), "kind": kind,
            "sample": sample, "seconds": dt}


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    r = reference_cpu(args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * r["seconds"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(r["cores"]) + " (CPU: one chain per core)",
                   "chains": r["cores"]},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"],
                         "kind": r["kind"], "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ GPU arm
def make_engine(dq, chains, seed0, precision, device=0, delay_rank=KB, ctas_per_sm=0,
                sweep_order=0, green_log=0, chain_ctas=0):
    T, bp = dq.square_lattice(LX, LX)
    eng = dq.Engine(device=device, precision=precision, delay_rank=delay_rank,
                    ctas_per_sm=ctas_per_sm, sweep_order=sweep_order, green_log=green_log,
                    chain_ctas=chain_ctas)
    m = eng.add_model(T, bp, U, DTAU, LX, LX, szz="af", sperp="af")
    for r in range(chains):
        eng.add_chain(m, L_SLICES, STAB, dq_replica_seed(SEED, 0, seed0 + r))
    return eng


def dq_replica_seed(base, b, r):
    """replica_seed (src/replica.c:17-34), as dqmc_host computes it."""
    import ctypes as C

    import dqmc_b200 as dq
    lib = dq.lib()
    lib.dqmc_replica_seed.restype = C.c_ulonglong
    lib.dqmc_replica_seed.argtypes = [C.c_ulonglong, C.c_int, C.c_int]
    return lib.dqmc_replica_seed(base, b, r)


def e2e_run(steps, warmup, chains, precision, device=0, seed=None):
    """The user-facing call end to end: dqmc_host_run on an input file for the
    same workload (host parsing, model exponential, uploads of the model and
    of every chain's field, initial G, warm-up and measured sweeps, read-back
    of the bins, jackknife and output files), wall-clock timed."""
    import ctypes as C

    import dqmc_b200 as dq
    lib = dq.lib()
    lib.dqmc_host_run.argtypes = [C.c_char_p]
    nbin = max(2, steps)
    nmeas = nbin * max(1, math.ceil(steps / nbin))
    text = (f"lattice=square\nLx={LX}\nLy={LX}\nbc=periodic\nt=-1.0\nU={U}\ndtau={DTAU}\n"
            f"beta_list={BETA}\nstab={STAB}\nnwarm={warmup}\nnmeas={nmeas}\nnbin={nbin}\n"
            f"nrep={chains}\nseed={SEED if seed is None else seed}\ndelay_rank={KB}\n"
            f"precision={precision}\ngpu_device={device}\n"
            f"replica_log=none\nszz_q=af\nsperp_q=af\n")
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input.txt"), "w") as f:
            f.write(text)
        os.chdir(d)
        try:
            devnull = os.open(os.devnull, os.O_WRONLY)
            saved = os.dup(1)
            os.dup2(devnull, 1)
            t0 = time.perf_counter()
            rc = lib.dqmc_host_run(b"input.txt")
            dt = time.perf_counter() - t0
            os.dup2(saved, 1)
            os.close(devnull)
            os.close(saved)
        finally:
            os.chdir(cwd)
    if rc != 0:
        return None
    sweeps = warmup + nmeas
    h2d = 3 * N_SITES * N_SITES * 8 + chains * (L_SLICES * N_SITES + 32)
    d2h = chains * nbin * (9 + 2) * 8
    return {"value": chains * N_SITES * L_SLICES * sweeps / dt, "unit": UNIT,
            "h2d_bytes_per_step": int(h2d / sweeps), "d2h_bytes_per_step": int(d2h / sweeps),
            "seconds": dt, "sweeps": sweeps,
            "note": "whole dqmc_gpu job (setup, uploads, initial G, warm-up and measured "
                    "sweeps, read-back, outputs) through dqmc_host_run; bytes are the job's "
                    "host<->device copies divided by its sweeps"}


def lockstep_check(dq, nchains=4, sweeps=2):
    """FP64 and mixed engines in lock step from the same seeds: field flips
    compared, and max|G_mixed - G_FP64| of G as wrapped just before every
    stabilization point (green_log snapshots; after a rebuild both are the
    same FP64 function of the field), beside each mode's stabilization drift
    max|G_wrapped - G_rebuilt| (the reference's drift diagnostic,
    src/dqmc.c:64-98, on the engine's own rebuild)."""
    M = -(-L_SLICES // STAB)
    cap = M * sweeps + 2
    ea = make_engine(dq, nchains, 0, dq.PREC_FP64, green_log=cap)
    eb = make_engine(dq, nchains, 0, dq.PREC_MIXED, green_log=cap)
    ea.prepare(1)
    eb.prepare(1)
    ea.sweep(sweeps)
    eb.sweep(sweeps)
    same = all(np.array_equal(ea.field(c), eb.field(c)) for c in range(nchains))
    per_point = []
    for c in range(nchains):
        ga, gb = ea.green_log(c), eb.green_log(c)
        k = min(len(ga), len(gb))
        per_point += [float(np.max(np.abs(ga[i] - gb[i]))) for i in range(k)]
    drift = {"fp64": max(ea.counters(c)["drift_max"] for c in range(nchains)),
             "mixed": max(eb.counters(c)["drift_max"] for c in range(nchains))}
    ea.close()
    eb.close()
    return {"chains": nchains, "sweeps": sweeps, "identical_flips": same,
            "stabilization_points": len(per_point),
            "max_dG_pre_rebuild": max(per_point) if per_point else None,
            "median_dG_pre_rebuild": float(np.median(per_point)) if per_point else None,
            "bound": 1e-8,
            "stabilization_drift_max": drift}


def precision_compare(dq, chains, args, precision, value):
    """The other precision mode on the same workload (same chains, warm-up
    and timed sweeps), and the lock-step accuracy check."""
    other = dq.PREC_FP64 if precision == dq.PREC_MIXED else dq.PREC_MIXED
    e = make_engine(dq, chains, 0, other)
    e.prepare(1)
    for _ in range(args.warmup):
        e.sweep(1)
    e.sync()
    p0 = [e.profile(c) for c in range(chains)] if other == dq.PREC_MIXED else None
    e.mark(0)
    e.sweep(args.steps)
    e.mark(1)
    ms = e.elapsed_ms() / args.steps
    split = None
    if p0 is not None:
        p1 = [e.profile(c) for c in range(chains)]
        wrap_cyc = sum(p1[c]["wrap"] - p0[c]["wrap"] for c in range(chains)) / (chains * args.steps)
        flush_cyc = sum(p1[c]["flush"] - p0[c]["flush"] for c in range(chains)) / (chains * args.steps)
        # one split product of n x n by n x n: 36 digit products (p + q <= 7 of
        # 8 digits), n^3 int8 multiply-adds each; the wrap is two per slice
        ops = 2 * L_SLICES * 36 * 2 * N_SITES ** 3
        import torch
        nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        peak = INT8_DENSE_OPS / (nsm * SM_MAX_MHZ * 1e6)
        split = {"phase": "wrap (both split products and their digit splits and epilogues)",
                 "bound": "tensor (int8)", "int8_ops_per_chain_sweep": ops,
                 "wrap_cycles_per_chain_sweep": wrap_cyc,
                 "flush_cycles_per_chain_sweep": flush_cyc,
                 "achieved_ops_per_cycle_per_sm": ops / wrap_cyc,
                 "peak_ops_per_cycle_per_sm": peak, "frac": ops / wrap_cyc / peak,
                 "peak_source": "nominal dense int8 4.5 POPS / (SMs x 1965 MHz); one chain "
                                "per SM, phase clocks of each chain"}
    e.close()
    other_value = chains * N_SITES * L_SLICES / (ms * 1e-3)
    fp64_v, mixed_v = (value, other_value) if precision == dq.PREC_FP64 else (other_value, value)
    return {"fp64_value": fp64_v, "mixed_value": mixed_v, "mixed_over_fp64": mixed_v / fp64_v,
            "target_ratio": 3.0,
            "mixed": "wrap and delayed-update flush as FP64-emulated int8 split products "
                     "(8 balanced base-256 digits per line, tcgen05.mma kind::i8, exact int32 "
                     "accumulation in tensor memory); QR, G from UDV, B-blocks, ratios FP64",
            "split_roofline": split,
            "lockstep": lockstep_check(dq)}


def batch_line(dq, kind, precision, sweeps, peak, tuned=False):
    """One of the batched workloads as a sub-line: 'uneven' = the 64-chain
    mix of 4x4..12x12 lattices with drawn U and beta (one launch per sweep,
    bounded by its most expensive chain), 'lowt' = 8 chains of 24x24, U=8,
    dtau=0.05, beta=10 (L=200), stab 5, delay rank 64.  Field updates/s over
    timed sweeps after one untimed sweep, device-timed; roofline on the
    chains' algorithmic FLOPs against the measured DGEMM peak."""
    from dqmc_b200.workloads import LOWT, uneven_batch
    tuning = None
    if kind == "uneven":
        chains = [dict(w, stab=8) for w in uneven_batch()]
        if tuned:
            # per size class: delay rank, flush grouping and interval
            # (the workload leaves n_wrap to the tuner), dqmc_b200.autotune
            from dqmc_b200 import autotune
            keys = sorted({(w["Lx"], w["L"], w["U"]) for w in chains})
            classes = [dict(Lx=Lx, Ly=Lx, n=Lx * Lx, L=L, U=U_, dtau=DTAU, stab=8)
                       for Lx, L, U_ in keys]
            t0 = time.perf_counter()
            tuner = autotune.Tuner()
            picks = dict(zip(keys, tuner.tune(classes, tune_stab=True)))
            tuning = {"seconds": time.perf_counter() - t0, "trials": tuner.trials,
                      "classes": len(keys),
                      "choices": {f"{Lx}x{Lx} L={L} U={U_:g}": {k: p[k] for k in
                                  ("delay_rank", "flush_pairs", "stab")}
                                  for (Lx, L, U_), p in picks.items()}}
            for w in chains:
                p = picks[(w["Lx"], w["L"], w["U"])]
                w.update(stab=p["stab"], delay_rank=p["delay_rank"],
                         flush_pairs=p["flush_pairs"])
        eng = dq.Engine(precision=precision)
    else:
        chains = [dict(Lx=LOWT["Lx"], n=LOWT["Lx"] ** 2, U=LOWT["U"], dtau=LOWT["dtau"],
                       L=LOWT["L"], stab=LOWT["stab"], seed=s) for s in LOWT["seeds"]]
        eng = dq.Engine(precision=precision, delay_rank=LOWT["delay_rank"])
    models = {}
    for w in chains:
        key = (w["Lx"], w["U"], w["dtau"])
        if key not in models:
            T, bp = dq.square_lattice(w["Lx"], w["Lx"])
            models[key] = eng.add_model(T, bp, w["U"], w["dtau"], w["Lx"], w["Lx"])
        cid = eng.add_chain(models[key], w["L"], w["stab"], w["seed"])
        if "delay_rank" in w:
            eng.tune_chain(cid, w["delay_rank"], w["flush_pairs"])
    t0 = time.perf_counter()
    eng.prepare(1)
    eng.sweep(1)
    eng.sync()
    setup_s = time.perf_counter() - t0
    c0 = [eng.counters(c) for c in range(len(chains))]
    eng.mark(0)
    eng.sweep(sweeps)
    eng.mark(1)
    ms = eng.elapsed_ms() / sweeps
    c1 = [eng.counters(c) for c in range(len(chains))]
    _, chain_ctas, cluster_chains = eng.residency()
    eng.close()
    upd = sum(w["n"] * w["L"] for w in chains)
    flops = sum(flops_per_chain_sweep(w["n"], w["L"], w["stab"],
                                      (c1[i]["accepted"] - c0[i]["accepted"]) / sweeps)
                for i, w in enumerate(chains))
    achieved = flops / (ms * 1e-3) / 1e12
    crit = max(chains, key=lambda w: w["n"] ** 3 * w["L"])
    crit_line = {"n": crit["n"], "L": crit["L"]}
    if not tuned and (kind == "uneven" or precision == dq.PREC_FP64):
        # the most expensive chain alone: a launch of one chain per CTA
        # cannot take less than this chain's own sweep
        e1 = dq.Engine(precision=precision,
                       delay_rank=LOWT["delay_rank"] if kind == "lowt" else 0)
        T, bp = dq.square_lattice(crit["Lx"], crit["Lx"])
        m1 = e1.add_model(T, bp, crit["U"], crit["dtau"], crit["Lx"], crit["Lx"])
        e1.add_chain(m1, crit["L"], crit["stab"], crit["seed"])
        e1.prepare(1)
        e1.sweep(1)
        e1.sync()
        e1.mark(0)
        e1.sweep(sweeps)
        e1.mark(1)
        alone = e1.elapsed_ms() / sweeps
        alone_ctas = e1.residency()[1]
        e1.close()
        crit_line.update(ms_per_sweep_alone=alone, batch_over_alone=ms / alone,
                         chain_ctas_alone=alone_ctas)
    line = {"value": upd / (ms * 1e-3), "unit": UNIT, "ms_per_sweep": ms, "sweeps": sweeps,
            "chains": len(chains), "field_updates_per_sweep": upd,
            "precision": "mixed" if precision == dq.PREC_MIXED else "fp64",
            "chains_failed": sum(1 for c in c1 if c["status"] != 0),
            "chain_ctas": chain_ctas, "chains_on_a_cluster": cluster_chains,
            "setup_and_first_sweep_s": setup_s,
            "critical_chain": crit_line,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "flops_per_launch": flops}}
    if tuning:
        line["autotune"] = tuning
    return line


def c3_sigma(dq, nwarm=100, nmeas=400, nbin=20):
    """The single-chain 16x16 workload as specified (seed 11, nwarm 100,
    nmeas 400, 20 bins) in FP64 and in mixed precision: each observable's
    jackknife mean and error per mode, and |mean_mixed - mean_fp64| in units
    of the FP64 error bar."""
    out = {}
    res = {}
    for prec, name in ((dq.PREC_FP64, "fp64"), (dq.PREC_MIXED, "mixed")):
        T, bp = dq.square_lattice(LX, LX)
        e = dq.Engine(precision=prec, delay_rank=KB)
        m = e.add_model(T, bp, U, DTAU, LX, LX, szz="af", sperp="af")
        e.add_chain(m, L_SLICES, STAB, SEED)
        e.prepare(nbin)
        e.sweep(nwarm)
        per = nmeas // nbin
        for b in range(nbin):
            e.sweep_measure(per, b)
        sc, zz, pp = e.bins(0)
        e.close()
        sgn = sc[:, 5]
        cols = {"E_hub": sc[:, 0] / sgn, "E_gc": sc[:, 1] / sgn, "n": sc[:, 3] / sgn,
                "D": sc[:, 4] / sgn, "Szz_af": zz[:, 0] / sgn, "Sperp_af": pp[:, 0] / sgn}
        res[name] = {}
        for k, x in cols.items():
            x = np.asarray(x)
            loo = (x.sum() - x) / (len(x) - 1)
            err = math.sqrt((len(x) - 1) / len(x) * np.sum((loo - loo.mean()) ** 2))
            res[name][k] = (float(x.mean()), err)
    for k in res["fp64"]:
        m64, e64 = res["fp64"][k]
        mmx, emx = res["mixed"][k]
        out[k] = {"fp64": [m64, e64], "mixed": [mmx, emx],
                  "diff_in_sigma": abs(mmx - m64) / e64 if e64 > 0 else None}
    return {"workload": "16x16 U=4 beta=8, one chain, seed 11, nwarm 100, nmeas 400, 20 bins",
            "observables": out}


def alternating_order(dq, chains, args, precision, value):
    """The same workload in sweep_order=alternating (forward sweeps carrying
    the prefix stack, backward sweeps rebuilding the suffix stack): timed
    over an even number of sweeps after the same warm-up."""
    e = make_engine(dq, chains, 0, precision, sweep_order=dq.SWEEP_ALTERNATING)
    e.prepare(1)
    for _ in range(max(4, args.warmup + (args.warmup & 1))):
        e.sweep(1)
    e.sync()
    k = max(2, args.steps + (args.steps & 1))
    e.mark(0)
    e.sweep(k)
    e.mark(1)
    ms = e.elapsed_ms() / k
    e.close()
    v = chains * N_SITES * L_SLICES / (ms * 1e-3)
    return {"value": v, "unit": UNIT, "ms_per_sweep": ms, "over_forward": v / value,
            "sweeps": k}


def run_gpu_arm(args):
    import torch
    import torch.distributed as dist

    import dqmc_b200 as dq
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    os.environ.setdefault("CUDA_DEVICE_ORDER", "PCI_BUS_ID")
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    props = torch.cuda.get_device_properties(local)
    chains = args.chains or 2 * props.multi_processor_count
    precision = dq.PREC_MIXED if args.precision == "mixed" else dq.PREC_FP64
    eng = make_engine(dq, chains, rank * chains, precision, device=local,
                      ctas_per_sm=args.ctas_per_sm, chain_ctas=args.chain_ctas)
    nbin = max(1, args.steps)
    eng.prepare(nbin)
    per_sm, chain_ctas, cluster_chains = eng.residency()
    for w in range(args.warmup):
        eng.sweep_measure(1, 0)
    eng.sync()
    eng.clear_bins()
    c0 = [eng.counters(c) for c in range(chains)]

    def barrier():
        if world > 1:
            t = torch.zeros(1, device="cuda")
            dist.all_reduce(t)
            torch.cuda.synchronize()

    sampler = ClockSampler(physical_gpu_index(local))
    barrier()
    eng.sync()
    eng.kernel_timing(True)
    eng.mark(0)
    for k in range(args.steps):
        eng.sweep_measure(1, k % nbin)
    eng.mark(1)
    ms = eng.elapsed_ms()
    eng.sync()
    barrier()
    clocks = sampler.stop()
    sweep_ms, nsweep, meas_ms, nmeas = eng.kernel_times()
    eng.kernel_timing(False)
    c1 = [eng.counters(c) for c in range(chains)]
    status_bad = sum(1 for c in c1 if c["status"] != 0)
    accepted = sum(c1[i]["accepted"] - c0[i]["accepted"] for i in range(chains))
    attempts = sum(c1[i]["attempts"] - c0[i]["attempts"] for i in range(chains))
    drift = max(c["drift_max"] for c in c1)
    drifts = np.array([c["drift_max"] for c in c1])
    ms_max = ms
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * chains * N_SITES * L_SLICES * args.steps / (ms_max * 1e-3)
    eng.close()

    # end to end through the public entry point on every rank (its own
    # device and seeds), the slowest rank's wall time
    e2e = None
    if not args.no_e2e:
        barrier()
        r = e2e_run(args.steps, args.warmup, chains, args.precision, device=local,
                    seed=SEED + 1000 * rank)
        dt = r["seconds"] if r else float("inf")
        if world > 1:
            t = torch.tensor([dt], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        if r and math.isfinite(dt):
            e2e = dict(r, value=world * r["value"] * r["seconds"] / dt, seconds=dt)

    if rank == 0:
        acc_per_chain_sweep = accepted / max(1, chains * args.steps)
        flops_launch = chains * flops_per_chain_sweep(N_SITES, L_SLICES, STAB, acc_per_chain_sweep)
        exec_launch = chains * executed_flops_per_chain_sweep(N_SITES, L_SLICES, STAB,
                                                              acc_per_chain_sweep)
        avg_launch = sweep_ms / max(1, nsweep)
        achieved = flops_launch / (avg_launch * 1e-3) / 1e12
        peak, peak_src = 40.0, "nominal B200 FP64 tensor (DGEMM probe skipped)"
        if not args.no_peak:
            try:
                peak = fp64_gemm_peak_tflops()
                peak_src = "measured: cuBLAS DGEMM 8192^3 on this GPU (bench.py)"
            except Exception as exc:  # pragma: no cover
                peak_src = f"nominal B200 FP64 tensor (DGEMM probe failed: {exc})"
        tb = traffic_per_chain_sweep(precision == dq.PREC_MIXED)
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak,
                    "unit": "TFLOP/s", "frac": achieved / peak,
                    "traffic": tb * chains if tb else None,
                    "traffic_gbs": tb * chains / (avg_launch * 1e-3) / 1e9 if tb else None,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                      "k_sweep launch of 296 chains (profiles/), per chain-sweep "
                                      "x chains",
                    "kernel": "k_sweep (one launch = one sweep of every chain)",
                    "flops_per_launch": flops_launch,
                    "flops_definition": "algorithmic F(measured acceptance) per chain-sweep "
                                        "x chains (reference algorithm)",
                    "executed_flops_per_launch": exec_launch,
                    "executed_tflops": exec_launch / (avg_launch * 1e-3) / 1e12,
                    "avg_launch_ms": avg_launch,
                    "peak_source": peak_src}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if precision == dq.PREC_FP64 else "f64 (split i8 wrap/flush)",
            "data": "synthetic: HS fields drawn from each chain's own xoshiro256** stream",
            "config": {"workload": workload_name(chains), "chains_per_gpu": chains,
                       "n": N_SITES, "L": L_SLICES, "stab": STAB, "delay_rank": KB,
                       "precision": args.precision,
                       "residency": {"chains_per_sm": per_sm, "cluster_ctas": chain_ctas,
                                     "chains_on_a_cluster": cluster_chains},
                       "l2": f"inputs larger than L2: {chains} chains x ~21 MB resident "
                             f"state >> {L2_BYTES // 2**20} MB L2",
                       "parallelism": f"replicas x{world} (no collective on the data path)"},
            "roofline": roofline,
            "gpu_launches": nsweep + nmeas,
            "clocks": clocks,
            "acceptance": accepted / max(1, attempts),
            "drift_max": drift,
            "drift": {"definition": "per chain, max|G_wrapped - G_rebuilt| over its "
                                    "stabilization points in the timed sweeps",
                      "median": float(np.median(drifts)),
                      "p99": float(np.percentile(drifts, 99)), "max": float(drifts.max())},
            "chains_failed": status_bad,
            "measure_ms_per_step": meas_ms / max(1, nmeas),
        }
        if world == 1 and not args.no_workloads:
            line["workloads"] = {
                "uneven_batch_64": dict(
                    {p: batch_line(dq, "uneven", pv, 3, peak)
                     for p, pv in (("fp64", dq.PREC_FP64), ("mixed", dq.PREC_MIXED))},
                    fp64_tuned=batch_line(dq, "uneven", dq.PREC_FP64, 3, peak, tuned=True)),
                "lowt_24x24_beta10": {p: batch_line(dq, "lowt", pv, 1, peak)
                                      for p, pv in (("fp64", dq.PREC_FP64),
                                                    ("mixed", dq.PREC_MIXED))}}
        if world == 1 and args.c3_sigma:
            line["c3_sigma"] = c3_sigma(dq)
        if world == 1 and not args.no_compare:
            line["precision_compare"] = precision_compare(dq, chains, args, precision, value)
            line["alternating_order"] = alternating_order(dq, chains, args, precision, value)
        if not args.no_single_chain and world == 1:
            # one chain: a thread-block cluster per chain (automatic size)
            # and, for comparison, one CTA per chain; same trajectory
            single = {}
            for key, cc, prec in (("cluster", 0, precision), ("one_cta", 1, precision),
                                  ("mixed_cluster", 0, dq.PREC_MIXED)):
                e1 = make_engine(dq, 1, 0, prec, chain_ctas=cc)
                e1.prepare(1)
                e1.sweep(1)
                e1.sync()
                e1.mark(0)
                e1.sweep(2)
                e1.mark(1)
                single[key] = (e1.elapsed_ms() / 2, e1.residency()[1])
                e1.close()
            t1, cc1 = single["cluster"]
            line["single_chain"] = {"value": N_SITES * L_SLICES / (t1 * 1e-3), "unit": UNIT,
                                    "ms_per_sweep": t1, "chain_ctas": cc1,
                                    "one_cta_ms_per_sweep": single["one_cta"][0],
                                    "over_one_cta": single["one_cta"][0] / t1,
                                    "mixed_ms_per_sweep": single["mixed_cluster"][0],
                                    "mixed_chain_ctas": single["mixed_cluster"][1]}
        if e2e is not None:
            line["e2e"] = e2e
        if not args.no_cpu_baseline and world == 1:
            cb = reference_cpu(2, 0)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--chains", type=int, default=0, help="chains per GPU (0: 2 x SMs)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the other precision mode and the same-seed check")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-single-chain", action="store_true")
    ap.add_argument("--no-peak", action="store_true", help="skip the DGEMM peak probe")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the uneven-batch and low-temperature sub-lines")
    ap.add_argument("--c3-sigma", action="store_true",
                    help="also run the single-chain 100/400/20 workload in both precisions "
                         "and report each observable's difference in FP64 error bars")
    ap.add_argument("--chain-ctas", type=int, default=0,
                    help="CTAs per chain of the main line's engine (0: automatic)")
    ap.add_argument("--ctas-per-sm", type=int, default=0, choices=[0, 1, 2],
                    help="sweep kernel residency (0: automatic)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)   # at least three untimed steps
    from dqmc_b200 import launch
    if args.gpus > 1 and not launch.under_launcher():
        # one rank per GPU, as torchrun would start them (rank 0 prints)
        sys.exit(launch.main_self(args.gpus))
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
