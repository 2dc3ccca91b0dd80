"""Host driver pieces (no GPU): input parsing and validation, lattices, spin
plans, replica seeds, jackknife, bin ratios, sum rules and the 14-column
row format, each against the reference's behaviour."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, golden

dq = pytest.importorskip("dqmc_b200")


class Params(C.Structure):
    _fields_ = [("lattice", C.c_char * 16), ("latfile", C.c_char * 256),
                ("Lx", C.c_int), ("Ly", C.c_int), ("pbc", C.c_int),
                ("thop", C.c_double), ("U", C.c_double), ("dtau", C.c_double),
                ("beta_list", C.c_double * 64), ("nbeta", C.c_int),
                ("nwarm", C.c_int), ("nmeas", C.c_int), ("nbin", C.c_int),
                ("stab_interval", C.c_int), ("output_file", C.c_char * 256),
                ("profile", C.c_int), ("profile_file", C.c_char * 256),
                ("stab_drift_file", C.c_char * 256), ("udv_scale_file", C.c_char * 256),
                ("udv_centered_file", C.c_char * 256), ("sweep_order", C.c_char * 16),
                ("green_rebuild", C.c_char * 16), ("parallel", C.c_char * 16),
                ("nrep", C.c_int), ("replica_log", C.c_char * 256),
                ("szz_q", C.c_char * 256), ("szz_file", C.c_char * 256),
                ("sperp_q", C.c_char * 256), ("sperp_file", C.c_char * 256),
                ("spin_consistency_file", C.c_char * 256), ("seed", C.c_ulonglong),
                ("delay_rank", C.c_int), ("precision", C.c_char * 16),
                ("gpu_device", C.c_int), ("gpu_devices", C.c_int * 16), ("ngpu", C.c_int)]


class Lattice(C.Structure):
    _fields_ = [("n", C.c_int), ("Lx", C.c_int), ("Ly", C.c_int), ("type", C.c_int),
                ("has_coordinates", C.c_int), ("is_bipartite", C.c_int),
                ("t", C.POINTER(C.c_double)), ("bipart", C.POINTER(C.c_int))]


class Plan(C.Structure):
    _fields_ = [("enabled", C.c_int), ("is_all", C.c_int), ("n", C.c_int),
                ("Lx", C.c_int), ("Ly", C.c_int), ("nq", C.c_int),
                ("mx", C.POINTER(C.c_int)), ("my", C.POINTER(C.c_int))]


@pytest.fixture(scope="module")
def L():
    lib = dq.lib()
    lib.dqmc_params_read.argtypes = [C.POINTER(Params), C.c_char_p]
    lib.dqmc_replica_seed.restype = C.c_ulonglong
    lib.dqmc_replica_seed.argtypes = [C.c_ulonglong, C.c_int, C.c_int]
    lib.dqmc_jackknife.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.dqmc_bin_values.argtypes = [C.c_void_p, C.c_void_p]
    lib.dqmc_format_row.argtypes = [C.c_char_p, C.c_size_t, C.c_double] + [C.c_void_p] * 7 + [C.c_int]
    lib.dqmc_sum_rule.argtypes = [C.POINTER(Plan), C.c_void_p, C.c_double, C.c_double,
                                  C.c_double, C.c_void_p, C.c_void_p]
    return lib


def read(L, tmp_path, text):
    f = tmp_path / "in.txt"
    f.write_text(text)
    p = Params()
    rc = L.dqmc_params_read(C.byref(p), str(f).encode())
    return rc, p


def test_reference_inputs_parse(L, tmp_path):
    rc, p = read(L, tmp_path, "lattice=chain\nLx=4\npbc=1\nt=-1.0\nU=4.0\ndtau=0.1\n"
                 "beta_list=0.5,1.0,2.0,4.0,6.0,8.0\nnwarm=300\nnmeas=3000\nnbin=30\nseed=1\n")
    assert rc == 0
    assert p.lattice == b"chain" and p.Lx == 4 and p.nbeta == 6
    assert list(p.beta_list[:6]) == [0.5, 1.0, 2.0, 4.0, 6.0, 8.0]
    assert (p.nwarm, p.nmeas, p.nbin, p.seed, p.stab_interval) == (300, 3000, 30, 1, 8)
    assert p.output_file == b"observables.dat" and p.szz_q == b"none"


def test_defaults_and_engine_keys(L, tmp_path):
    rc, p = read(L, tmp_path, "# only comments\n\nU = 7\n")   # 'U = 7' is not key=value
    assert rc == 0 and p.U == 4.0 and p.nbeta == 1 and p.beta_list[0] == 2.0
    rc, p = read(L, tmp_path, "delay_rank=16\nprecision=mixed\ngpu_device=0\n")
    assert rc == 0 and p.delay_rank == 16 and p.precision == b"mixed" and p.ngpu == 0
    rc, p = read(L, tmp_path, "gpu_devices=0,3,1\n")
    assert rc == 0 and p.ngpu == 3 and list(p.gpu_devices)[:3] == [0, 3, 1]
    for bad in ("gpu_devices=0,-1\n", "gpu_devices=a\n", "gpu_devices=" + ",".join(["0"] * 17) + "\n"):
        assert read(L, tmp_path, bad)[0] == 1


def test_replica_ownership_matches_reference(L):
    """The reference's own vectors for its MPI replica split
    (tests/test_mpi_replica.c:27-66)."""
    L.dqmc_replica_rank_range.argtypes = [C.c_int] * 3 + [C.POINTER(C.c_int)] * 2
    L.dqmc_replica_gather_layout.argtypes = [C.c_int] * 4 + [C.c_void_p] * 2
    first, count = C.c_int(), C.c_int()

    def rr(nrep, nranks, rank):
        L.dqmc_replica_rank_range(nrep, nranks, rank, C.byref(first), C.byref(count))
        return first.value, count.value

    assert [rr(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    assert [rr(2, 4, r) for r in range(4)] == [(0, 1), (1, 1), (2, 0), (2, 0)]
    owners = {(10, 3, 0): 0, (10, 3, 3): 0, (10, 3, 4): 1, (10, 3, 7): 2, (2, 4, 0): 0,
              (2, 4, 1): 1, (10, 3, 10): -1, (0, 2, 0): -1}
    for args, want in owners.items():
        assert L.dqmc_replica_rank_for_replica(*args) == want
    rc, dp = np.zeros(4, np.int32), np.zeros(4, np.int32)
    assert L.dqmc_replica_gather_layout(5, 2, 3, 8, rc.ctypes.data, dp.ctypes.data) == 0
    assert list(rc[:3]) == [32, 32, 16] and list(dp[:3]) == [0, 32, 64]
    assert L.dqmc_replica_gather_layout(2 ** 31 - 1, 2, 1, 2, rc.ctypes.data, dp.ctypes.data) != 0


@pytest.mark.parametrize("text", ["bogus=1\n", "nbin=1\n", "nmeas=10\nnbin=3\n", "U=-1\n",
                                  "beta_list=1,-2\n", "bc=weird\n", "szz_q=a b\n",
                                  "sweep_order=sideways\n", "delay_rank=99\n"])
def test_invalid_inputs_rejected(L, tmp_path, text):
    rc, _ = read(L, tmp_path, text)
    assert rc == 1


def test_replica_seed_and_jackknife(L):
    g = golden("rng")
    for args, want in zip(g["replica_args"], g["replica_seeds"]):
        assert L.dqmc_replica_seed(*(int(a) for a in args)) == int(want)
    x = np.ascontiguousarray(g["jk_x"])
    m, e = C.c_double(), C.c_double()
    L.dqmc_jackknife(x.ctypes.data, len(x), C.byref(m), C.byref(e))
    assert m.value == g["jk"][0] and abs(e.value - g["jk"][1]) < 1e-15


def test_bin_values_and_row_format(L):
    # one bin: sums of sign*value over 4 samples with sign = 1
    b = np.array([-4.0, -8.0, -6.0, 8.0, 0.5, 4.0, 4.0, 30.0, 40.0])
    out = np.zeros(6)
    assert L.dqmc_bin_values(b.ctypes.data, out.ctypes.data) == 0
    np.testing.assert_allclose(out, [-1.0, -2.0, -1.5, 2.0, 0.125, 1.0])
    bad = b.copy()
    bad[5] = 0.0
    assert L.dqmc_bin_values(bad.ctypes.data, out.ctypes.data) == 1
    series = [np.array(v, dtype=np.float64) for v in
              ([1.0, 3.0, 5.0], [2.0] * 3, [0.0] * 3, [4.0] * 3, [0.1] * 3, [1.0] * 3, [0.5] * 3)]
    buf = C.create_string_buffer(512)
    assert L.dqmc_format_row(buf, 512, 0.25, *[s.ctypes.data for s in series], 3) == 0
    # src/main.c:259-262 format
    want = "%.6g %.8g %.3g %.8g %.3g %.8g %.3g %.6g %.2g %.8g %.2g %.6g %.8g %.3g\n" % (
        0.25, 3.0, np.sqrt(4 / 3), 2.0, 0.0, 0.0, 0.0, 4.0, 0.0, 0.1, 0.0, 1.0, 0.5, 0.0)
    assert buf.value.decode() == want


def test_lattice_and_plans(L, tmp_path):
    lib = L
    lib.dqmc_lattice_square.argtypes = [C.POINTER(Lattice), C.c_int, C.c_int, C.c_double, C.c_int]
    lib.dqmc_lattice_file.argtypes = [C.POINTER(Lattice), C.c_char_p]
    lib.dqmc_lattice_free.argtypes = [C.POINTER(Lattice)]
    lib.dqmc_spin_plan.argtypes = [C.POINTER(Plan), C.POINTER(Lattice), C.c_char_p]
    lib.dqmc_spin_plan_free.argtypes = [C.POINTER(Plan)]
    g = golden("sq4_b4")
    lat = Lattice()
    assert lib.dqmc_lattice_square(C.byref(lat), 4, 4, -1.0, 1) == 0
    T = np.ctypeslib.as_array(lat.t, shape=(16 * 16,)).reshape(16, 16).T
    np.testing.assert_array_equal(T, g["thop"])
    # lattice=file round trip with BFS two-colouring
    f = tmp_path / "lat.txt"
    f.write_text("16\n" + "\n".join(" ".join("%.17g" % v for v in row) for row in g["thop"]) + "\n")
    lat2 = Lattice()
    assert lib.dqmc_lattice_file(C.byref(lat2), str(f).encode()) == 0
    assert lat2.is_bipartite == 1 and lat2.has_coordinates == 0
    bp = np.ctypeslib.as_array(lat2.bipart, shape=(16,))
    np.testing.assert_array_equal(bp, g["bipart"])
    plan = Plan()
    assert lib.dqmc_spin_plan(C.byref(plan), C.byref(lat), b"af") == 0
    assert plan.nq == 1 and plan.mx[0] == 2 and plan.my[0] == 2
    lib.dqmc_spin_plan_free(C.byref(plan))
    assert lib.dqmc_spin_plan(C.byref(plan), C.byref(lat), b"0:0,1:3") == 0 and plan.nq == 2
    lib.dqmc_spin_plan_free(C.byref(plan))
    for sel in (b"4:0", b"0:0,0:0", b"1:1,", b"x"):
        assert lib.dqmc_spin_plan(C.byref(plan), C.byref(lat), sel) == 1
    assert lib.dqmc_spin_plan(C.byref(plan), C.byref(lat2), b"af") == 1   # no coordinates
    assert lib.dqmc_spin_plan(C.byref(plan), C.byref(lat), b"all") == 0 and plan.is_all
    # sum rule: sum_q Szz = 1/4 (ntot - 2 n D)
    vals = np.full(16, 0.25 * (16 - 2 * 16 * 0.1) / 16)
    assert lib.dqmc_sum_rule(C.byref(plan), vals.ctypes.data, 16.0, 0.1, 0.25, None, None) == 0
    vals[0] += 1e-6
    assert lib.dqmc_sum_rule(C.byref(plan), vals.ctypes.data, 16.0, 0.1, 0.25, None, None) == 1
    lib.dqmc_spin_plan_free(C.byref(plan))
    lib.dqmc_lattice_free(C.byref(lat))
    lib.dqmc_lattice_free(C.byref(lat2))


@pytest.mark.parametrize("extra,msg", [
    ("udv_scale_file=s.dat\nparallel=omp\n", "udv_scale_file currently supports parallel=serial only"),
    ("udv_centered_file=c.dat\nparallel=omp\n",
     "udv_centered_file currently supports parallel=serial only"),
    ("udv_centered_file=c.dat\n", "udv_centered_file requires green_rebuild=centered"),
])
def test_driver_rejects_diagnostics_like_reference(tmp_path, extra, msg):
    """The reference's checks on the UDV diagnostic files (src/main.c:733-762),
    made before any device work."""
    import subprocess
    exe = os.path.join(ROOT, "sai-qmc_b200", "dqmc_gpu")
    if not os.path.exists(exe):
        pytest.skip("dqmc_gpu not built")
    (tmp_path / "input.txt").write_text("lattice=chain\nLx=4\npbc=1\n" + extra)
    r = subprocess.run([exe, "input.txt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and msg in r.stderr
