"""Python mirror of the engine's C ABI (include/dqmc_gpu.h) via ctypes.

The compute path is the CUDA library ``libdqmc_b200.so``; this module only
moves host buffers in and out.  Importing it never falls back to a CPU path:
``Engine`` raises if the library or a CUDA device is missing.

The chain-level names follow the reference's sweep-engine seam
(SAI-QMC src/dqmc.h:91-108): ``sweep`` = dqmc_sweep, counters =
accept_attempts / accept_accepted / sweep_count / status / sign.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("DQMC_B200_LIB") or os.path.join(PKG, "libdqmc_b200.so")

PREC_FP64, PREC_MIXED = 0, 1
SWEEP_FORWARD, SWEEP_ALTERNATING = 0, 1
REBUILD_COMBINE, REBUILD_TWO_SIDED, REBUILD_CENTERED = 0, 1, 2
DRIFT_STAB, DRIFT_SCRATCH = 1, 2
PAIRS_AUTO, PAIRS_OFF, PAIRS_ON = 0, 1, 2
UDV_DIRECTIONS = ["stack_suffix_pre_rmul", "stack_prefix_pre_lmul", "forward", "backward",
                  "left_udv_forward", "left_udv_backward"]
UDV_RECORD_DOUBLES = 16
BIN_FIELDS = ["sum_sign_Ehub", "sum_sign_Egc", "sum_sign_Eph", "sum_sign_N",
              "sum_sign_D", "sum_sign", "count", "accepted", "attempts"]
NBIN_FIELDS = len(BIN_FIELDS)
PHASES = ["bcache", "stack", "propose", "flush", "wrap", "bblock", "lmul",
          "combine", "green", "sdrift", "adopt", "measure"]

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


class Desc(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int),
                ("delay_rank", C.c_int), ("drift", C.c_int),
                ("ctas_per_sm", C.c_int), ("sweep_order", C.c_int), ("green_rebuild", C.c_int),
                ("flush_pairs", C.c_int), ("udv_diag", C.c_int), ("green_log", C.c_int),
                ("chain_ctas", C.c_int), ("cluster_chains", C.c_int)]


class Counters(C.Structure):
    _fields_ = [("attempts", C.c_ulonglong), ("accepted", C.c_ulonglong),
                ("sweeps", C.c_ulonglong), ("status", C.c_int), ("pad", C.c_int),
                ("sign", C.c_double), ("drift_max", C.c_double),
                ("drift_mean", C.c_double), ("drift_samples", C.c_ulonglong),
                ("scratch_drift_max", C.c_double),
                ("scratch_drift_mean", C.c_double),
                ("scratch_drift_samples", C.c_ulonglong),
                ("scratch_drift_max_tau", C.c_int), ("pad2", C.c_int),
                ("scratch_drift_max_sweep", C.c_ulonglong),
                ("rng", C.c_uint64 * 4)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("pad", "pad2", "rng")}
        d["rng"] = np.array(list(self.rng), dtype=np.uint64)
        return d


_lib = None


def lib():
    """Load libdqmc_b200.so (raises OSError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    L = C.CDLL(LIB_PATH)
    L.dqmc_last_error.restype = C.c_char_p
    L.dqmc_desc_default.argtypes = [C.POINTER(Desc)]
    L.dqmc_engine_create.restype = C.c_void_p
    L.dqmc_engine_create.argtypes = [C.POINTER(Desc)]
    L.dqmc_engine_destroy.argtypes = [C.c_void_p]
    L.dqmc_model_add.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, _ip,
                                 C.c_double, C.c_double]
    L.dqmc_model_add_mu.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, C.c_void_p,
                                    C.c_double, C.c_double, C.c_int, C.c_double, C.c_int]
    L.dqmc_read_green_down.argtypes = [C.c_void_p, C.c_int, _dp]
    L.dqmc_model_set_spin.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.dqmc_chain_add.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                 C.c_uint64, C.c_void_p]
    L.dqmc_engine_prepare.argtypes = [C.c_void_p, C.c_int]
    L.dqmc_chain_tune.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.dqmc_sweep.argtypes = [C.c_void_p, C.c_int]
    L.dqmc_sweep_measure.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.dqmc_synchronize.argtypes = [C.c_void_p]
    L.dqmc_chain_count.argtypes = [C.c_void_p]
    L.dqmc_engine_residency.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int)]
    L.dqmc_read_green.argtypes = [C.c_void_p, C.c_int, _dp]
    L.dqmc_read_field.argtypes = [C.c_void_p, C.c_int, _bp]
    L.dqmc_write_field.argtypes = [C.c_void_p, C.c_int, _bp]
    L.dqmc_read_counters.argtypes = [C.c_void_p, C.c_int, C.POINTER(Counters)]
    L.dqmc_read_bins.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                 C.c_void_p]
    L.dqmc_clear_bins.argtypes = [C.c_void_p]
    L.dqmc_read_profile.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    L.dqmc_kernel_timing.argtypes = [C.c_void_p, C.c_int]
    L.dqmc_kernel_times.argtypes = [C.c_void_p] + [C.c_void_p] * 4
    L.dqmc_timer_mark.argtypes = [C.c_void_p, C.c_int]
    L.dqmc_timer_elapsed.argtypes = [C.c_void_p, C.c_void_p]
    L.dqmc_green_from_scratch.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp,
                                          C.POINTER(C.c_int)]
    L.dqmc_wrap_green.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
    L.dqmc_udv_green.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp,
                                 C.POINTER(C.c_int)]
    L.dqmc_udv_green2.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp,
                                  C.c_double, _dp, C.POINTER(C.c_int)]
    L.dqmc_write_green.argtypes = [C.c_void_p, C.c_int, _dp]
    L.dqmc_write_rng.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_uint64)]
    L.dqmc_expm_sym.argtypes = [C.c_int, _dp, C.c_double, _dp]
    L.dqmc_read_udv_records.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    L.dqmc_read_green_log.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    L.dqmc_udv_green_noalloc.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp,
                                         C.POINTER(C.c_int)]
    _lib = L
    return L


class DqmcError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise DqmcError(f"{what}: {lib().dqmc_last_error().decode()}")


def _cm(A):
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T).ravel()


def _from_cm(buf, n):
    return buf.reshape(n, n).T.copy()


def square_lattice(Lx, Ly, t=-1.0, pbc=True):
    """Hopping matrix and bipartite signs of lattice_square (src/lattice.c:46-82)."""
    n = Lx * Ly
    T = np.zeros((n, n))
    bp = np.zeros(n, dtype=np.int32)
    for y in range(Ly):
        for x in range(Lx):
            i = x + y * Lx
            if x + 1 < Lx:
                j = (x + 1) + y * Lx
            elif pbc and Lx > 1:
                j = y * Lx
            else:
                j = -1
            if j >= 0:
                T[i, j] += t
                T[j, i] += t
            if y + 1 < Ly:
                j = x + (y + 1) * Lx
            elif pbc and Ly > 1:
                j = x
            else:
                j = -1
            if j >= 0:
                T[i, j] += t
                T[j, i] += t
            bp[i] = 1 if (x + y) % 2 == 0 else -1
    return T, bp


def chain_lattice(Lx, t=-1.0, pbc=True):
    """Hopping matrix and bipartite signs of lattice_chain (src/lattice.c:26-44)."""
    T = np.zeros((Lx, Lx))
    bp = np.zeros(Lx, dtype=np.int32)
    for x in range(Lx):
        if x + 1 < Lx:
            j = x + 1
        elif pbc and Lx > 1:
            j = 0
        else:
            j = -1
        if j >= 0:
            T[x, j] += t
            T[j, x] += t
        bp[x] = 1 if x % 2 == 0 else -1
    return T, bp


def q_list(Lx, Ly, selector):
    """(mx, my) lists of structure_factor_plan_init selectors none/af/all."""
    if selector == "none":
        return [], []
    if selector == "af":
        return [Lx // 2 if Lx > 1 else 0], [Ly // 2 if Ly > 1 else 0]
    if selector == "all":
        mx, my = [], []
        for y in range(Ly):
            for x in range(Lx):
                mx.append(x)
                my.append(y)
        return mx, my
    raise ValueError(selector)


class Engine:
    """A batch of chains on one GPU (the C ABI's dqmc_engine)."""

    def __init__(self, device=0, precision=PREC_FP64, delay_rank=0,
                 drift=DRIFT_STAB, ctas_per_sm=0, sweep_order=SWEEP_FORWARD,
                 green_rebuild=REBUILD_COMBINE, flush_pairs=PAIRS_AUTO, udv_diag=0,
                 green_log=0, chain_ctas=0, cluster_chains=0):
        L = lib()
        d = Desc()
        L.dqmc_desc_default(C.byref(d))
        d.device, d.precision, d.delay_rank, d.drift = device, precision, delay_rank, drift
        d.ctas_per_sm = ctas_per_sm
        d.sweep_order = sweep_order
        d.green_rebuild = green_rebuild
        d.flush_pairs = flush_pairs
        d.udv_diag = udv_diag
        d.green_log = green_log
        d.chain_ctas = chain_ctas
        d.cluster_chains = cluster_chains
        self.green_log_cap = green_log
        self.h = L.dqmc_engine_create(C.byref(d))
        if not self.h:
            raise DqmcError(L.dqmc_last_error().decode())
        self.models = []
        self.chains = []
        self.nbin = 0

    def add_model(self, thop, bipart, U, dtau, Lx=0, Ly=0, szz="none",
                  sperp="none", mu=None, two_spin=False):
        """mu=None: half filling (mu = U/2).  bipart=None (non-bipartite
        lattice), a mu off half filling or two_spin=True: the two-spin path
        (G_up and G_down evolved separately)."""
        thop = np.asarray(thop, dtype=np.float64)
        n = thop.shape[0]
        bp = None if bipart is None else np.ascontiguousarray(bipart, dtype=np.int32)
        self._bp = bp
        mid = lib().dqmc_model_add_mu(self.h, n, Lx, Ly, _cm(thop),
                                      None if bp is None else bp.ctypes.data_as(C.c_void_p),
                                      U, dtau, 1 if mu is None else 0,
                                      0.0 if mu is None else float(mu), int(two_spin))
        if mid < 0:
            raise DqmcError(lib().dqmc_last_error().decode())
        zx, zy = q_list(Lx, Ly, szz) if szz != "none" else ([], [])
        px, py = q_list(Lx, Ly, sperp) if sperp != "none" else ([], [])
        if zx or px:
            arrs = [np.asarray(a, dtype=np.int32) for a in (zx, zy, px, py)]
            ptr = [a.ctypes.data_as(C.c_void_p) if len(a) else None for a in arrs]
            _check(lib().dqmc_model_set_spin(self.h, mid, len(zx), ptr[0], ptr[1],
                                             len(px), ptr[2], ptr[3]), "set_spin")
            self._keep = arrs
        self.models.append(dict(n=n, nq_zz=len(zx), nq_perp=len(px)))
        return mid

    def add_chain(self, model, L, stab, seed, field=None):
        fp = None
        if field is not None:
            fa = np.ascontiguousarray(np.asarray(field, dtype=np.int8).ravel())
            self._f = fa
            fp = fa.ctypes.data_as(C.c_void_p)
        cid = lib().dqmc_chain_add(self.h, model, L, stab, seed, fp)
        if cid < 0:
            raise DqmcError(lib().dqmc_last_error().decode())
        self.chains.append(dict(model=model, n=self.models[model]["n"], L=L))
        return cid

    def tune_chain(self, c, delay_rank, flush_pairs=PAIRS_AUTO):
        """Per-chain delay rank and flush grouping (before prepare)."""
        _check(lib().dqmc_chain_tune(self.h, c, delay_rank, flush_pairs), "chain_tune")

    def prepare(self, nbin=1):
        self.nbin = nbin
        _check(lib().dqmc_engine_prepare(self.h, nbin), "prepare")

    def sweep(self, k=1):
        _check(lib().dqmc_sweep(self.h, k), "sweep")

    def sweep_measure(self, k, bin):
        _check(lib().dqmc_sweep_measure(self.h, k, bin), "sweep_measure")

    def sync(self):
        _check(lib().dqmc_synchronize(self.h), "synchronize")

    def green(self, c):
        n = self.chains[c]["n"]
        g = np.zeros(n * n)
        _check(lib().dqmc_read_green(self.h, c, g), "read_green")
        return _from_cm(g, n)

    def green_down(self, c):
        n = self.chains[c]["n"]
        g = np.zeros(n * n)
        _check(lib().dqmc_read_green_down(self.h, c, g), "read_green_down")
        return _from_cm(g, n)

    def field(self, c):
        ch = self.chains[c]
        f = np.zeros(ch["n"] * ch["L"], dtype=np.int8)
        _check(lib().dqmc_read_field(self.h, c, f), "read_field")
        return f.reshape(ch["L"], ch["n"])

    def write_field(self, c, field):
        f = np.ascontiguousarray(np.asarray(field, dtype=np.int8).ravel())
        _check(lib().dqmc_write_field(self.h, c, f), "write_field")

    def write_green(self, c, G):
        _check(lib().dqmc_write_green(self.h, c, _cm(np.asarray(G, dtype=np.float64))),
               "write_green")

    def write_rng(self, c, rng):
        a = (C.c_uint64 * 4)(*[int(x) for x in rng])
        _check(lib().dqmc_write_rng(self.h, c, a), "write_rng")

    def counters(self, c):
        out = Counters()
        _check(lib().dqmc_read_counters(self.h, c, C.byref(out)), "read_counters")
        return out.as_dict()

    def bins(self, c):
        m = self.models[self.chains[c]["model"]]
        sc = np.zeros(self.nbin * NBIN_FIELDS)
        zz = np.zeros(max(1, self.nbin * m["nq_zz"]))
        pp = np.zeros(max(1, self.nbin * m["nq_perp"]))
        _check(lib().dqmc_read_bins(self.h, c, sc.ctypes.data_as(C.c_void_p),
                                    zz.ctypes.data_as(C.c_void_p),
                                    pp.ctypes.data_as(C.c_void_p)), "read_bins")
        return (sc.reshape(self.nbin, NBIN_FIELDS),
                zz[: self.nbin * m["nq_zz"]].reshape(self.nbin, m["nq_zz"]),
                pp[: self.nbin * m["nq_perp"]].reshape(self.nbin, m["nq_perp"]))

    def green_log(self, c):
        """Snapshots of the chain's G as wrapped, just before each
        stabilization point since the last call (needs green_log > 0):
        array (k, n, n)."""
        n = self.chains[c]["n"]
        cap = max(1, self.green_log_cap)
        buf = np.zeros(cap * n * n)
        k = lib().dqmc_read_green_log(self.h, c, buf.ctypes.data, cap)
        if k < 0:
            raise DqmcError(lib().dqmc_last_error().decode())
        return np.stack([_from_cm(buf[i * n * n:(i + 1) * n * n], n) for i in range(k)]) \
            if k else np.zeros((0, n, n))

    def udv_records(self, c):
        """The chain's UDV scale records since the last call (needs
        udv_diag=1): rows of UDV_RECORD_DOUBLES, see include/dqmc_gpu.h."""
        out = []
        buf = np.zeros(256 * UDV_RECORD_DOUBLES)
        while True:
            k = lib().dqmc_read_udv_records(self.h, c, buf.ctypes.data, 256)
            if k < 0:
                raise DqmcError(lib().dqmc_last_error().decode())
            if k == 0:
                break
            out.append(buf[: k * UDV_RECORD_DOUBLES].reshape(k, UDV_RECORD_DOUBLES).copy())
        return np.concatenate(out) if out else np.zeros((0, UDV_RECORD_DOUBLES))

    def profile(self, c):
        """Per-phase SM cycles of chain c (PHASES order)."""
        out = (C.c_ulonglong * len(PHASES))()
        _check(lib().dqmc_read_profile(self.h, c, out, len(PHASES)), "read_profile")
        return dict(zip(PHASES, [int(x) for x in out]))

    def kernel_timing(self, enable=True):
        _check(lib().dqmc_kernel_timing(self.h, int(enable)), "kernel_timing")

    def kernel_times(self):
        """(sweep ms, sweep launches, measure ms, measure launches)."""
        a, b, c, d = C.c_double(), C.c_int(), C.c_double(), C.c_int()
        _check(lib().dqmc_kernel_times(self.h, C.byref(a), C.byref(b), C.byref(c),
                                       C.byref(d)), "kernel_times")
        return a.value, b.value, c.value, d.value

    def mark(self, which):
        _check(lib().dqmc_timer_mark(self.h, which), "timer_mark")

    def elapsed_ms(self):
        ms = C.c_double()
        _check(lib().dqmc_timer_elapsed(self.h, C.byref(ms)), "timer_elapsed")
        return ms.value

    def residency(self):
        """(chains per SM, cluster size, chains on a cluster each) of the
        sweep kernel, as prepared."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib().dqmc_engine_residency(self.h, C.byref(a), C.byref(b), C.byref(c)),
               "residency")
        return a.value, b.value, c.value

    def clear_bins(self):
        _check(lib().dqmc_clear_bins(self.h), "clear_bins")

    def green_from_scratch(self, c, l0=0):
        n = self.chains[c]["n"]
        g = np.zeros(n * n)
        ds = C.c_int()
        _check(lib().dqmc_green_from_scratch(self.h, c, l0, g, C.byref(ds)),
               "green_from_scratch")
        return _from_cm(g, n), ds.value

    def wrap(self, c, l, G):
        n = self.chains[c]["n"]
        g = _cm(G)
        _check(lib().dqmc_wrap_green(self.h, c, l, g), "wrap_green")
        return _from_cm(g, n)

    def close(self):
        if getattr(self, "h", None):
            lib().dqmc_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def udv_green(U, D, T, device=0):
    """G = (1 + U diag(D) T)^{-1} on the device (dqmc_udv_green)."""
    n = U.shape[0]
    g = np.zeros(n * n)
    ds = C.c_int()
    _check(lib().dqmc_udv_green(device, n, _cm(U),
                                np.ascontiguousarray(D, dtype=np.float64), _cm(T), g,
                                C.byref(ds)), "udv_green")
    return _from_cm(g, n), ds.value


def udv_green2(UL, DL, TL, off_L, UR, DR, TR, off_R, device=0):
    """G = (1 + L R)^{-1} from two UDV factors scaled by exp(off) (T_R unit
    upper triangular), two-sided reconstruction (dqmc_udv_green2)."""
    n = UL.shape[0]
    g = np.zeros(n * n)
    ds = C.c_int()
    _check(lib().dqmc_udv_green2(device, n, _cm(UL), np.ascontiguousarray(DL, dtype=np.float64),
                                 _cm(TL), float(off_L), _cm(UR),
                                 np.ascontiguousarray(DR, dtype=np.float64), _cm(TR),
                                 float(off_R), g, C.byref(ds)), "udv_green2")
    return _from_cm(g, n), ds.value


def udv_green_noalloc(U, D, T, device=0):
    """As udv_green, through the entry point that allocates no device
    memory (fixed in-library scratch, n <= 128; dqmc_udv_green_noalloc)."""
    n = U.shape[0]
    g = np.zeros(n * n)
    ds = C.c_int()
    _check(lib().dqmc_udv_green_noalloc(device, n, _cm(U),
                                        np.ascontiguousarray(D, dtype=np.float64), _cm(T),
                                        g, C.byref(ds)), "udv_green_noalloc")
    return _from_cm(g, n), ds.value


def expm_sym(A, scale):
    """exp(scale*A) for symmetric A (host helper, dqmc_expm_sym)."""
    n = A.shape[0]
    out = np.zeros(n * n)
    _check(lib().dqmc_expm_sym(n, _cm(A), scale, out), "expm_sym")
    return _from_cm(out, n)
