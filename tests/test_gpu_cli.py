"""End-to-end: the dqmc_gpu driver on a reference input file.

With the same seeds the GPU chains flip exactly the same fields as the
reference, so observables.dat, szz.dat, sperp.dat and the consistency file
agree with the reference program to rounding (compared at 1e-6 relative
after the reference's own %.6g-%.8g printing), and with the CPU oracle.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

INPUT = """lattice=chain
Lx=4
pbc=1
t=-1.0
U=4.0
dtau=0.1
beta_list=0.5,1.0,2.0
nwarm=20
nmeas=40
nbin=4
nrep=2
seed=1
szz_q=all
sperp_q=all
spin_consistency_file=consistency.dat
"""

EXE = os.path.join(PKG, "dqmc_gpu")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "dqmc")


def run(exe, d, extra=""):
    (d / "input.txt").write_text(INPUT + extra)
    r = subprocess.run([exe, "input.txt"], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r


def table(path):
    rows = [l.split() for l in open(path) if l.strip() and not l.startswith("#")]
    return np.array([[float(x) for x in r] for r in rows])


def oracle_rows(oracle):
    """The same run through the CPU oracle: bins, ratios and jackknife."""
    beta, nwarm, nmeas, nbin, nrep, U = [0.5, 1.0, 2.0], 20, 40, 4, 2, 4.0
    rows = []
    for b, bt in enumerate(beta):
        L = int(round(bt / 0.1))
        series = [[] for _ in range(7)]
        for r in range(nrep):
            seed = oracle.replica_seed(1, b, r)
            ch = oracle.chain(0, 4, 1, U, 0.1, L, 8, seed)
            ch.sweep(nwarm)
            a0 = ch.state()
            for _ in range(nbin):
                acc = np.zeros(6)
                att0, acc0 = a0["attempts"], a0["accepted"]
                for _ in range(nmeas // nbin):
                    ch.sweep(1)
                    m, _, _ = oracle.measure(ch, 0)
                    E, ntot, D = m[0], m[3], m[4]
                    acc += [E, E - U / 2 * ntot, E - 0.5 * U * ntot + 0.25 * U * 4, ntot, D, 1.0]
                a0 = ch.state()
                cnt = nmeas // nbin
                vals = list(acc[:5] / acc[5]) + [acc[5] / cnt,
                                                 (a0["accepted"] - acc0) / (a0["attempts"] - att0)]
                for k in range(7):
                    series[k].append(vals[k])
        out = [1.0 / (L * 0.1)]
        for k, s in enumerate(series):
            m, e = oracle.jackknife(np.array(s))
            out += [m] if k == 5 else [m, e]
        rows.append(out)
    return np.array(rows)


def test_cli_matches_reference_and_oracle(tmp_path, oracle):
    gdir = tmp_path / "gpu"
    gdir.mkdir()
    run(EXE, gdir)
    obs = table(gdir / "observables.dat")
    assert obs.shape == (3, 14)
    # 14-column header and row format of the reference (src/main.c:909, 259-262)
    head = open(gdir / "observables.dat").read().splitlines()
    assert head[1].startswith("# T  E_hub dE_hub  E_gc dE_gc")
    want = oracle_rows(oracle)
    np.testing.assert_allclose(obs[:, [0, 1, 3, 5, 7, 9, 11, 12]],
                               want[:, [0, 1, 3, 5, 7, 9, 11, 12]], rtol=1e-6, atol=1e-9)
    for name in ("szz.dat", "sperp.dat", "consistency.dat"):
        t = table(gdir / name)
        assert t.shape == (3 * 4, 12)
    if os.path.exists(REF_EXE):
        rdir = tmp_path / "ref"
        rdir.mkdir()
        run(REF_EXE, rdir)
        for name in ("observables.dat", "szz.dat", "sperp.dat", "consistency.dat"):
            a, b = table(gdir / name), table(rdir / name)
            assert a.shape == b.shape
            np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-9, err_msg=name)
        ha = [l for l in open(gdir / "szz.dat") if l.startswith("#")]
        hb = [l for l in open(rdir / "szz.dat") if l.startswith("#")]
        assert ha == hb


def test_cli_rejects_like_reference(tmp_path):
    (tmp_path / "input.txt").write_text("lattice=chain\nLx=5\npbc=1\n")
    r = subprocess.run([EXE, "input.txt"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "non-bipartite" in r.stderr
    (tmp_path / "input.txt").write_text("beta_list=0.55\ndtau=0.1\nnmeas=4\nnbin=2\n")
    r = subprocess.run([EXE, "input.txt"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "not a multiple of dtau" in r.stderr


def test_cli_alternating_matches_reference(tmp_path):
    """sweep_order=alternating through the whole program: the same rows as
    the reference program's alternating run."""
    if not os.path.exists(REF_EXE):
        pytest.skip("reference program not built here")
    extra = "sweep_order=alternating\nstab=4\n"
    gdir, rdir = tmp_path / "gpu", tmp_path / "ref"
    gdir.mkdir()
    rdir.mkdir()
    run(EXE, gdir, extra)
    run(REF_EXE, rdir, extra)
    for name in ("observables.dat", "szz.dat", "sperp.dat", "consistency.dat"):
        a, b = table(gdir / name), table(rdir / name)
        assert a.shape == b.shape
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-9, err_msg=name)


def test_cli_replicas_split_over_devices(tmp_path):
    """gpu_devices: each listed device runs its contiguous replica range of
    every beta (the reference's MPI split, src/replica_mpi.c:13-37); two
    engines on the one device give the same outputs as one engine, and
    replicas.dat gains the owner column of the MPI runner."""
    one, two = tmp_path / "one", tmp_path / "two"
    one.mkdir()
    two.mkdir()
    extra = "nrep=3\nreplica_log=replicas.dat\n"
    run(EXE, one, extra)
    run(EXE, two, extra + "gpu_devices=0,0\n")
    for name in ("observables.dat", "szz.dat", "sperp.dat", "consistency.dat"):
        a = [l for l in open(one / name) if not l.startswith("#")]
        b = [l for l in open(two / name) if not l.startswith("#")]
        assert a == b, name
    ra = [l.split() for l in open(one / "replicas.dat") if not l.startswith("#")]
    rb = [l.split() for l in open(two / "replicas.dat") if not l.startswith("#")]
    assert len(ra) == len(rb) == 9
    for x, y in zip(ra, rb):
        assert len(x) == 8 and len(y) == 9 and x == y[:8]
        assert int(y[8]) == (0 if int(y[2]) < 2 else 1)


def prof_table(path):
    out = {}
    for l in open(path):
        if l.startswith("#"):
            continue
        x = l.split()
        assert len(x) == 14
        out[(x[0], x[4], x[5])] = (int(x[6]), float(x[7]), float(x[9]))
    return out


def test_cli_profile_file_like_reference(tmp_path):
    """profile=1: the reference's profile.dat rows (src/profiler.c:188-223).
    Region call counts that are fixed by the algorithm equal the reference
    program's; times are the engine's own (device cycles at the SM clock)."""
    g = tmp_path / "gpu"
    g.mkdir()
    run(EXE, g, "profile=1\n")
    head = open(g / "profile.dat").readline()
    assert head == ("# beta T dtau Ltr phase region calls total_sec avg_sec frac_beta wall_sec "
                    "thread_total_sec nrep parallel\n")
    t = prof_table(g / "profile.dat")
    betas = sorted({k[0] for k in t})
    assert len(betas) == 3
    for b in betas:
        bt = t[(b, "all", "beta_total")]
        assert bt[0] == 1 and bt[1] > 0
        for ph in ("warmup", "measurement"):
            assert t[(b, ph, "dqmc_sweep")][0] == 2 * (20 if ph == "warmup" else 40)
        for (bb, ph, reg), (calls, sec, frac) in t.items():
            if bb != b or reg == "beta_total":
                continue
            assert calls > 0 and sec >= 0 and abs(frac - sec / bt[1]) <= 1e-12 * max(1, frac)
            if ph == "all":
                parts = [t.get((b, p, reg), (0, 0.0, 0))[0]
                         for p in ("setup", "warmup", "measurement", "finalize")]
                assert calls == sum(parts)
    if os.path.exists(REF_EXE):
        r = tmp_path / "ref"
        r.mkdir()
        run(REF_EXE, r, "profile=1\n")
        assert open(r / "profile.dat").readline() == head
        ref = prof_table(r / "profile.dat")
        fixed = ("dqmc_sweep", "green_wrap", "measure_sample", "green_stack_build", "udv_lmul",
                 "udv_rmul", "udv_combine", "udv_inv_one_plus")
        n = 0
        for (b, ph, reg), v in ref.items():
            if ph in ("warmup", "measurement") and reg in fixed:
                assert t[(b, ph, reg)][0] == v[0], (b, ph, reg)
                n += 1
        assert n > 0
