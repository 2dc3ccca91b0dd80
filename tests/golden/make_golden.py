"""Generate the golden parity fixtures from the UNMODIFIED reference.

Run in a container where the reference sources exist (``$SAIQMC_REF``, else
a ``reference`` directory beside the repository):
``python tests/golden/make_golden.py``.  It
builds oracle/_ref (oracle/build.py), drives the reference engine through
oracle/ref_shim.c and writes small .npz files next to this script.  The
reference's own UDV fixtures (tests/fixtures/udv_phase6a_*.txt, read here as
data) are re-packed into udv_fixture.npz.  ``--only-alternating`` writes
just the sweep_order=alternating fixtures (*_alt.npz), ``--only-rebuild``
the green_rebuild=two_sided/centered ones, ``--only-two-spin`` the
two-spin (use_ph = 0) ones.  The GPU box never needs the
reference: tests read only the .npz files.
"""
from __future__ import annotations

import io
import os
import subprocess
import sys

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build as obuild  # noqa: E402
from oracle.bind import LAT_CHAIN, LAT_SQUARE, Reference  # noqa: E402

# the reference checkout: $SAIQMC_REF, else a "reference" directory beside
# the repository root (oracle/build.py uses the same rule)
REF = obuild.REF

# (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps, selector)
CASES = [
    ("chain4_b2", LAT_CHAIN, 4, 1, 4.0, 0.1, 20, 8, 1, 4, "all"),
    ("chain4_u0", LAT_CHAIN, 4, 1, 0.0, 0.1, 20, 8, 5, 2, "all"),
    ("sq4_b4", LAT_SQUARE, 4, 4, 4.0, 0.1, 40, 10, 7, 3, "all"),
    ("sq6_b2", LAT_SQUARE, 6, 6, 6.0, 0.1, 20, 8, 3, 3, "af"),
    ("sq8_b4", LAT_SQUARE, 8, 8, 4.0, 0.1, 40, 10, 7, 2, "af"),
]

# sweep_order=alternating (forward sweeps storing the prefix stack, backward
# sweeps with B^-1 G B wraps rebuilding the suffix stack): 4 sweeps each
# (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps)
ALT_CASES = [
    ("chain4_alt", LAT_CHAIN, 4, 1, 4.0, 0.1, 20, 8, 1, 4),
    ("sq4_b4_alt", LAT_SQUARE, 4, 4, 4.0, 0.1, 40, 10, 7, 4),
    ("sq6_b2_alt", LAT_SQUARE, 6, 6, 6.0, 0.1, 20, 8, 3, 4),
    ("sq8_b4_alt", LAT_SQUARE, 8, 8, 4.0, 0.1, 40, 10, 7, 4),
]
# green_rebuild=two_sided / centered (G from the two boundary factors):
# (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps, alternating, rebuild)
REBUILD_CASES = [
    ("sq4_b4_2s", LAT_SQUARE, 4, 4, 4.0, 0.1, 40, 10, 7, 3, False, 1),
    ("sq8_b4_2s", LAT_SQUARE, 8, 8, 4.0, 0.1, 40, 10, 7, 3, False, 1),
    ("chain4_ctr", LAT_CHAIN, 4, 1, 4.0, 0.1, 20, 8, 1, 3, False, 2),
    ("sq6_b2_2s_alt", LAT_SQUARE, 6, 6, 6.0, 0.1, 20, 8, 3, 4, True, 1),
]
# the two-spin path (use_ph = 0, dqmc.c:641-813): forced at the PH point,
# a non-bipartite chain at half filling, a doped square lattice
# (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps, half, mu, force)
TWO_SPIN_CASES = [
    ("sq4_2spin", LAT_SQUARE, 4, 4, 4.0, 0.1, 20, 5, 5, 3, 1, 0.0, 1),
    ("chain3_2spin", LAT_CHAIN, 3, 1, 4.0, 0.1, 10, 4, 19, 4, 1, 0.0, 0),
    ("sq4_mu", LAT_SQUARE, 4, 4, 4.0, 0.1, 20, 5, 7, 3, 0, 0.7, 0),
]
HEADLINE_ALT = dict(Lx=16, U=4.0, dtau=0.1, L=80, stab=8, base_seed=11, chains=2, sweeps=4)

# the headline lattice: 16x16 U=4 dtau=0.1 beta=8 stab=8, chains seeded as
# the benchmark's replicas (replica_seed(11, 0, r)); fields and drift only
HEADLINE = dict(Lx=16, U=4.0, dtau=0.1, L=80, stab=8, base_seed=11, chains=2, sweeps=3)


def _read_tokens(path):
    with open(path) as f:
        return f.read().split()


def udv_fixture(out):
    d = os.path.join(REF, "tests", "fixtures")
    tok = _read_tokens(os.path.join(d, "udv_phase6a_actual_n16.txt"))
    it = iter(tok)
    rec = {}
    key = None
    vals = []
    for t in it:
        try:
            vals.append(float(t))
        except ValueError:
            if key is not None:
                rec[key] = vals
            key, vals = t, []
    rec[key] = vals
    n = int(rec["n"][0])
    U = np.array(rec["U"]).reshape(n, n).T       # file is column-major
    D = np.array(rec["D"])
    T = np.array(rec["T"]).reshape(n, n).T
    gtok = _read_tokens(os.path.join(d, "udv_phase6a_actual_n16_green.txt"))
    ds = int(gtok[gtok.index("det_sign") + 1])
    g0 = gtok.index("G") + 1
    G = np.array([float(x) for x in gtok[g0:g0 + n * n]]).reshape(n, n).T
    np.savez_compressed(out, U=U, D=D, T=T, G=G, det_sign=ds,
                        offset=float(rec["offset"][0]),
                        min_logD=float(rec["min_logD"][0]),
                        max_logD=float(rec["max_logD"][0]))


def alternating(R):
    for (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps) in ALT_CASES:
        ch = R.chain(kind, Lx, Ly, U, dtau, L, stab, seed, drift=True, alternating=True)
        st0 = ch.state()
        fields, Gs, cnt = [], [], []
        for _ in range(sweeps):
            ch.sweep(1)
            st = ch.state()
            fields.append(st["field"])
            Gs.append(st["Gu"])
            cnt.append([st["attempts"], st["accepted"], st["sweeps"], st["status"]])
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            params=np.array([kind, Lx, Ly, L, stab, seed, sweeps], dtype=np.int64),
            U=U, dtau=dtau, field0=st0["field"], G0=st0["Gu"], fields=np.array(fields),
            Gs=np.array(Gs), counters=np.array(cnt, dtype=np.int64), drift=R.drift(ch),
            rng_end=st["rng"])
        ch.free()
    h = HEADLINE_ALT
    seeds, fields, drifts, cnts, Gend = [], [], [], [], []
    for r in range(h["chains"]):
        seed = R.replica_seed(h["base_seed"], 0, r)
        ch = R.chain(LAT_SQUARE, h["Lx"], h["Lx"], h["U"], h["dtau"], h["L"], h["stab"], seed,
                     drift=True, alternating=True)
        fr = []
        for _ in range(h["sweeps"]):
            ch.sweep(1)
            fr.append(ch.state()["field"])
        st = ch.state()
        seeds.append(seed)
        fields.append(fr)
        drifts.append(R.drift(ch))
        cnts.append([st["attempts"], st["accepted"]])
        Gend.append(st["Gu"][:8, :8])
        ch.free()
    # the same chains with 4 BLAS threads (a rounding variant of the same
    # reference): chain 0's first backward sweep meets an acceptance decision
    # at the rounding level (slice 17, site 236), which the variant takes the
    # other way; both trajectories are the reference's
    var = subprocess.run([sys.executable, __file__, "--headline-alt-fields"], check=True,
                         capture_output=True, env=dict(os.environ, OPENBLAS_NUM_THREADS="4"))
    variant = np.load(io.BytesIO(var.stdout))
    np.savez_compressed(os.path.join(HERE, "sq16_b8_alt.npz"), fields_t4=variant,
                        params=np.array([h["Lx"], h["L"], h["stab"], h["sweeps"]]),
                        U=h["U"], dtau=h["dtau"], seeds=np.array(seeds, dtype=np.uint64),
                        fields=np.array(fields), drift=np.array(drifts),
                        counters=np.array(cnts, dtype=np.int64), G_corner=np.array(Gend))


def rebuild_modes(R):
    for (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps, alt, rb) in REBUILD_CASES:
        ch = R.chain(kind, Lx, Ly, U, dtau, L, stab, seed, drift=True, alternating=alt,
                     rebuild=rb)
        st0 = ch.state()
        fields, Gs, cnt = [], [], []
        for _ in range(sweeps):
            ch.sweep(1)
            st = ch.state()
            fields.append(st["field"])
            Gs.append(st["Gu"])
            cnt.append([st["attempts"], st["accepted"], st["sweeps"], st["status"]])
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            params=np.array([kind, Lx, Ly, L, stab, seed, sweeps, int(alt), rb], dtype=np.int64),
            U=U, dtau=dtau, field0=st0["field"], fields=np.array(fields), Gs=np.array(Gs),
            counters=np.array(cnt, dtype=np.int64), drift=R.drift(ch), rng_end=st["rng"])
        ch.free()
    # the reference's two-sided fixture (tests/fixtures/udv_phase6a_two_sided_n4.txt)
    tok = _read_tokens(os.path.join(REF, "tests", "fixtures", "udv_phase6a_two_sided_n4.txt"))
    rec, key, vals = {}, None, []
    for t in tok:
        try:
            vals.append(float(t))
        except ValueError:
            if key is not None:
                rec[key] = vals
            key, vals = t, []
    rec[key] = vals
    n = int(rec["n"][0])
    cm = lambda v: np.array(v).reshape(n, n).T        # noqa: E731 (file is column-major)
    np.savez_compressed(os.path.join(HERE, "udv_two_sided_fixture.npz"),
                        UL=cm(rec["left_U"]), DL=np.array(rec["left_D"]), TL=cm(rec["left_T"]),
                        off_L=rec["left_offset"][0], UR=cm(rec["right_U"]),
                        DR=np.array(rec["right_D"]), TR=cm(rec["right_T"]),
                        off_R=rec["right_offset"][0], G=cm(rec["G"]),
                        det_sign=int(rec["det_sign"][0]))


def two_spin(R):
    for (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps, half, mu, force) in TWO_SPIN_CASES:
        ch = R.chain_mu(kind, Lx, Ly, U, dtau, L, stab, seed, half=bool(half), mu=mu,
                        two_spin=bool(force))
        st0 = ch.state()
        fields, Gu, Gd, cnt, sign, meas = [], [], [], [], [], []
        for _ in range(sweeps):
            ch.sweep(1)
            st = ch.state()
            fields.append(st["field"])
            Gu.append(st["Gu"])
            Gd.append(st["Gd"])
            sign.append(st["sign"])
            cnt.append([st["attempts"], st["accepted"], st["sweeps"], st["status"]])
            m, _, _ = R.measure(ch, None)
            meas.append(m)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            params=np.array([kind, Lx, Ly, L, stab, seed, sweeps, half, force], dtype=np.int64),
            U=U, dtau=dtau, mu=mu, field0=st0["field"], Gu0=st0["Gu"], Gd0=st0["Gd"],
            sign0=st0["sign"], fields=np.array(fields), Gu=np.array(Gu), Gd=np.array(Gd),
            sign=np.array(sign), counters=np.array(cnt, dtype=np.int64), meas=np.array(meas),
            rng_end=st["rng"])
        ch.free()


# The batched uneven workload (dqmc_b200.workloads.uneven_batch, 64 chains of
# 4x4..12x12 with drawn U and beta): a selection covering every lattice size,
# each run by the reference on its own (beta index 0 keeps the seed), 2 sweeps
# at stab 8.  And the large low-temperature lattice (workloads.LOWT, 24x24,
# U=8, dtau=0.05): the full beta=10 (L=200) for one sweep, and a short L=40
# for two sweeps.
BATCH_SELECTION = (0, 6, 12, 18, 24, 33, 49, 63)
BATCH_STAB, BATCH_SWEEPS = 8, 2


def _g_summary(G):
    """A full G for n <= 64; else its 32 x 32 corner, every 7th row/column
    and its Frobenius norm (fixtures stay small)."""
    n = G.shape[0]
    if n <= 64:
        return dict(G=G)
    return dict(G_corner=G[:32, :32], G_sub=G[::7, ::7], G_fro=np.linalg.norm(G))


def batch_fields():
    """Fields of the selected batch chains after each sweep, as .npy on
    stdout (run with another OPENBLAS_NUM_THREADS: a rounding variant of the
    same reference)."""
    sys.path.insert(0, os.path.join(ROOT, "sai-qmc_b200"))
    from dqmc_b200.workloads import uneven_batch
    R = Reference()
    chains = uneven_batch()
    out = []
    for c in BATCH_SELECTION:
        w = chains[c]
        ch = R.chain(LAT_SQUARE, w["Lx"], w["Lx"], w["U"], w["dtau"], w["L"], BATCH_STAB,
                     w["seed"], drift=True)
        fr = []
        for _ in range(BATCH_SWEEPS):
            ch.sweep(1)
            fr.append(ch.state()["field"].ravel())
        out.append(np.concatenate(fr))
        ch.free()
    buf = io.BytesIO()
    np.save(buf, np.concatenate(out))
    sys.stdout.buffer.write(buf.getvalue())


def batches(R):
    sys.path.insert(0, os.path.join(ROOT, "sai-qmc_b200"))
    from dqmc_b200.workloads import LOWT, uneven_batch
    chains = uneven_batch()
    out = dict(selection=np.array(BATCH_SELECTION), stab=BATCH_STAB, sweeps=BATCH_SWEEPS)
    for c in BATCH_SELECTION:
        w = chains[c]
        ch = R.chain(LAT_SQUARE, w["Lx"], w["Lx"], w["U"], w["dtau"], w["L"], BATCH_STAB,
                     w["seed"], drift=True)
        st0 = ch.state()
        fields, cnt = [], []
        for _ in range(BATCH_SWEEPS):
            ch.sweep(1)
            st = ch.state()
            fields.append(st["field"])
            cnt.append([st["attempts"], st["accepted"], st["sweeps"], st["status"]])
        out[f"field0_{c}"] = st0["field"]
        out[f"fields_{c}"] = np.array(fields)
        out[f"counters_{c}"] = np.array(cnt, dtype=np.int64)
        out[f"rng_{c}"] = st["rng"]
        for k, v in _g_summary(st["Gu"]).items():
            out[f"{k}_{c}"] = v
        ch.free()
    # the same chains with 4 BLAS threads: chain 24 (12x12, U=6, beta=10)
    # meets an acceptance decision at the rounding level in its second sweep
    # that the two thread counts take opposite ways; both are the reference's
    var = subprocess.run([sys.executable, __file__, "--batch-fields"], check=True,
                         capture_output=True, env=dict(os.environ, OPENBLAS_NUM_THREADS="4"))
    flat = np.load(io.BytesIO(var.stdout))
    off = 0
    for c in BATCH_SELECTION:
        sz = BATCH_SWEEPS * chains[c]["L"] * chains[c]["n"]
        out[f"fields_t4_{c}"] = flat[off:off + sz].reshape(out[f"fields_{c}"].shape)
        off += sz
    np.savez_compressed(os.path.join(HERE, "batch64_sel.npz"), **out)
    w = LOWT
    lo = {}
    for tag, L, seed, sweeps in (("full", w["L"], w["seeds"][0], 1),
                                 ("short", 40, w["seeds"][1], 2)):
        ch = R.chain(LAT_SQUARE, w["Lx"], w["Lx"], w["U"], w["dtau"], L, w["stab"], seed,
                     drift=True)
        st0 = ch.state()
        for k, v in _g_summary(st0["Gu"]).items():
            lo[f"{tag}_{k}0"] = v
        fields, cnt = [], []
        for _ in range(sweeps):
            ch.sweep(1)
            st = ch.state()
            fields.append(st["field"])
            cnt.append([st["attempts"], st["accepted"], st["sweeps"], st["status"]])
        lo[f"{tag}_params"] = np.array([w["Lx"], L, w["stab"], seed, sweeps], dtype=np.int64)
        lo[f"{tag}_field0"] = st0["field"]
        lo[f"{tag}_fields"] = np.array(fields)
        lo[f"{tag}_counters"] = np.array(cnt, dtype=np.int64)
        lo[f"{tag}_rng"] = st["rng"]
        lo[f"{tag}_drift"] = R.drift(ch)
        for k, v in _g_summary(st["Gu"]).items():
            lo[f"{tag}_{k}"] = v
        ch.free()
        # the reference's own consistency at this point: its two-spin path
        # builds G_down from the sigma = -1 factors, which must equal the
        # particle-hole map I - P G_up^T P of G_up at half filling
        cm = R.chain_mu(LAT_SQUARE, w["Lx"], w["Lx"], w["U"], w["dtau"], L, w["stab"], seed,
                        half=True, two_spin=True)
        sm = cm.state()
        p = np.array([1.0 if ((i % w["Lx"]) + (i // w["Lx"])) % 2 == 0 else -1.0
                      for i in range(w["Lx"] ** 2)])
        lo[f"{tag}_ref_ph_violation0"] = float(np.max(np.abs(
            sm["Gd"] - (np.eye(len(p)) - (p[:, None] * sm["Gu"].T) * p[None, :]))))
        cm.free()
    np.savez_compressed(os.path.join(HERE, "sq24_lowt.npz"), U=w["U"], dtau=w["dtau"], **lo)


def ed_table():
    """Rows of the reference's exact-diagonalization table for the 4-site
    U=4 chain (columns T, E_gc, C, N, Sz, S2, D_total, Z;
    data/benchmark_L468_U4_full_diag_20260626/README.md) at the temperatures
    the checks use."""
    path = os.path.join(REF, "data", "benchmark_L468_U4_full_diag_20260626", "reference",
                        "L4_U4_FullDiag.dat")
    rows = np.array([[float(x) for x in l.split()] for l in open(path) if l.strip()])
    want = [0.1, 0.15, 0.2, 0.25, 0.5, 1.0, 2.0]
    sel = np.array([rows[np.argmin(np.abs(rows[:, 0] - T))] for T in want])
    assert np.allclose(sel[:, 0], want)
    np.savez_compressed(os.path.join(HERE, "ed_chain4_u4.npz"), T=sel[:, 0], E_gc=sel[:, 1],
                        N=sel[:, 3], D_total=sel[:, 6], U=4.0, mu=2.0, L=4)


def headline_alt_fields():
    """Fields of the alternating headline chains, written as .npy to stdout."""
    R = Reference()
    h = HEADLINE_ALT
    out = []
    for r in range(h["chains"]):
        seed = R.replica_seed(h["base_seed"], 0, r)
        ch = R.chain(LAT_SQUARE, h["Lx"], h["Lx"], h["U"], h["dtau"], h["L"], h["stab"], seed,
                     drift=True, alternating=True)
        fr = []
        for _ in range(h["sweeps"]):
            ch.sweep(1)
            fr.append(ch.state()["field"])
        out.append(fr)
        ch.free()
    buf = io.BytesIO()
    np.save(buf, np.array(out))
    sys.stdout.buffer.write(buf.getvalue())


def main():
    if "--headline-alt-fields" in sys.argv:
        headline_alt_fields()
        return
    if "--batch-fields" in sys.argv:
        batch_fields()
        return
    obuild.build_ref()
    R = Reference()
    if "--only-alternating" in sys.argv:
        alternating(R)
        print("wrote alternating fixtures")
        return
    if "--only-two-spin" in sys.argv:
        two_spin(R)
        print("wrote two-spin fixtures")
        return
    if "--only-ed" in sys.argv:
        ed_table()
        print("wrote ed_chain4_u4.npz")
        return
    if "--only-batches" in sys.argv:
        batches(R)
        print("wrote batch64_sel.npz, sq24_lowt.npz")
        return
    if "--only-rebuild" in sys.argv:
        rebuild_modes(R)
        print("wrote green_rebuild fixtures")
        return
    # RNG streams and replica seeds (rng.c:17-37, replica.c:17-34)
    seeds = np.array([1, 7, 11, 12345, 2**63 + 5], dtype=np.uint64)
    draws = np.stack([R.rng(int(s), 16) for s in seeds])
    rs = [(12345, 0, 0), (12345, 3, 0), (12345, 0, 1), (12345, 2, 7), (1, 5, 3)]
    rseed = np.array([R.replica_seed(*t) for t in rs], dtype=np.uint64)
    jk_x = np.array([1.0, 3.0, 5.0, 2.5, -1.0])
    jk = np.array(R.jackknife(jk_x))
    np.savez_compressed(os.path.join(HERE, "rng.npz"), seeds=seeds, draws=draws,
                        replica_args=np.array(rs, dtype=np.int64), replica_seeds=rseed,
                        jk_x=jk_x, jk=jk)
    for (name, kind, Lx, Ly, U, dtau, L, stab, seed, sweeps, sel) in CASES:
        ch = R.chain(kind, Lx, Ly, U, dtau, L, stab, seed, drift=True)
        model = R.model(ch)
        st0 = ch.state()
        rc, gs, ds = ch.green_scratch(0)
        # one wrap of the initial G at slice 0
        gw = ch.wrap(0, st0["Gu"])
        fields, Gs, cnt, meas, szz, sperp = [], [], [], [], [], []
        for _ in range(sweeps):
            ch.sweep(1)
            st = ch.state()
            fields.append(st["field"])
            Gs.append(st["Gu"])
            cnt.append([st["attempts"], st["accepted"], st["sweeps"], st["status"]])
            m, z, p = R.measure(ch, sel)
            meas.append(m)
            szz.append(z)
            sperp.append(p)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            params=np.array([kind, Lx, Ly, L, stab, seed, sweeps], dtype=np.int64),
            U=U, dtau=dtau, selector=sel,
            expK=model["expK"], expKinv=model["expKinv"], thop=model["thop"],
            bipart=model["bipart"], field0=st0["field"], G0=st0["Gu"],
            G_scratch=gs, det_sign=ds, G_wrap0=gw,
            fields=np.array(fields), Gs=np.array(Gs),
            counters=np.array(cnt, dtype=np.int64), meas=np.array(meas),
            szz=np.array(szz), sperp=np.array(sperp), drift=R.drift(ch),
            rng_end=st["rng"])
        ch.free()
    h = HEADLINE
    seeds, fields, drifts, cnts, Gend = [], [], [], [], []
    for r in range(h["chains"]):
        seed = R.replica_seed(h["base_seed"], 0, r)
        ch = R.chain(LAT_SQUARE, h["Lx"], h["Lx"], h["U"], h["dtau"], h["L"], h["stab"], seed,
                     drift=True)
        fr = []
        for _ in range(h["sweeps"]):
            ch.sweep(1)
            fr.append(ch.state()["field"])
        st = ch.state()
        seeds.append(seed)
        fields.append(fr)
        drifts.append(R.drift(ch))
        cnts.append([st["attempts"], st["accepted"]])
        Gend.append(st["Gu"][:8, :8])
        ch.free()
    np.savez_compressed(os.path.join(HERE, "sq16_b8.npz"),
                        params=np.array([h["Lx"], h["L"], h["stab"], h["sweeps"]]),
                        U=h["U"], dtau=h["dtau"], seeds=np.array(seeds, dtype=np.uint64),
                        fields=np.array(fields), drift=np.array(drifts),
                        counters=np.array(cnts, dtype=np.int64), G_corner=np.array(Gend))
    udv_fixture(os.path.join(HERE, "udv_fixture.npz"))
    alternating(R)
    rebuild_modes(R)
    two_spin(R)
    batches(R)
    ed_table()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
