"""ctypes bindings for the CPU oracle (test infrastructure only).

``Oracle`` wraps ``oracle/liboracle.so`` (the plain-C restatement in
``oracle/oracle.c``); ``Reference`` wraps ``oracle/_ref/libdqmcref.so`` (the
unmodified reference engine behind ``oracle/ref_shim.c``), which exists only
where ``oracle/build.py`` could compile the reference.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg
import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_bp = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")

LAT_CHAIN, LAT_SQUARE = 0, 1


def _fortran(a, n):
    """Column-major n x n buffer -> numpy array indexed [i, j]."""
    return np.asarray(a).reshape(n, n).T.copy()


class _Chain:
    """Common chain accessors over either library."""

    def __init__(self, lib, prefix, handle, n, L):
        self._lib, self._p, self.h, self.n, self.L = lib, prefix, handle, n, L

    def _f(self, name):
        return getattr(self._lib, self._p + name)

    def sweep(self, k=1):
        return self._f("chain_sweep")(self.h, k)

    def state(self):
        n, L = self.n, self.L
        gu = np.zeros(n * n)
        gd = np.zeros(n * n)
        field = np.zeros(n * L, dtype=np.int8)
        cnt = np.zeros(3, dtype=np.uint64)
        rng = np.zeros(4, dtype=np.uint64)
        sign = C.c_double()
        status = C.c_int()
        self._f("chain_state")(self.h, gu, gd, field, cnt, C.byref(sign),
                               C.byref(status), rng)
        return dict(Gu=_fortran(gu, n), Gd=_fortran(gd, n),
                    field=field.reshape(L, n), attempts=int(cnt[0]),
                    accepted=int(cnt[1]), sweeps=int(cnt[2]),
                    sign=sign.value, status=status.value, rng=rng)

    def green_scratch(self, l0=0):
        g = np.zeros(self.n * self.n)
        ds = C.c_int()
        rc = self._f("green_scratch")(self.h, l0, g, C.byref(ds))
        return rc, _fortran(g, self.n), ds.value

    def wrap(self, l, G):
        g = np.ascontiguousarray(np.asarray(G, dtype=np.float64).T).ravel()
        self._f("wrap")(self.h, l, g)
        return _fortran(g, self.n)

    def free(self):
        if self.h:
            self._f("chain_free")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Oracle:
    """The plain-C restatement (oracle/oracle.c)."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "liboracle.so")
        lib = C.CDLL(path)
        lib.orc_chain_new.restype = C.c_void_p
        lib.orc_chain_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_double, C.c_double, C.c_double,
                                      C.c_int, C.c_int, C.c_ulonglong,
                                      C.c_void_p, C.c_int, C.c_int]
        lib.orc_chain_sweep.argtypes = [C.c_void_p, C.c_int]
        lib.orc_chain_state.argtypes = [C.c_void_p, _dp, _dp, _bp, _up,
                                        C.c_void_p, C.c_void_p, _up]
        lib.orc_chain_model.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip, _dp]
        lib.orc_chain_drift.argtypes = [C.c_void_p, _dp]
        lib.orc_green_scratch.argtypes = [C.c_void_p, C.c_int, _dp, C.c_void_p]
        lib.orc_wrap.argtypes = [C.c_void_p, C.c_int, _dp]
        lib.orc_chain_measure.argtypes = [C.c_void_p, _dp, C.c_int, _dp, _dp]
        lib.orc_chain_free.argtypes = [C.c_void_p]
        lib.orc_udv_inv.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_void_p]
        lib.orc_expm_sym.argtypes = [C.c_int, _dp, C.c_double, _dp]
        lib.orc_replica_seed.restype = C.c_ulonglong
        lib.orc_replica_seed.argtypes = [C.c_ulonglong, C.c_int, C.c_int]
        lib.orc_jackknife.argtypes = [_dp, C.c_int, C.c_void_p, C.c_void_p]
        lib.orc_rng.argtypes = [C.c_ulonglong, C.c_int, _dp]
        lib.orc_measure_g.argtypes = [C.c_int, _dp, C.c_double, _dp, _dp, _dp]
        lib.orc_spin_g.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _dp,
                                   _dp, _dp, _dp]
        self.lib = lib

    def chain(self, kind, Lx, Ly, U, dtau, L, stab, seed, field=None,
              pbc=1, t=-1.0, delay=16, drift=False):
        n = Lx * (Ly if kind == LAT_SQUARE else 1)
        fp = None
        if field is not None:
            fa = np.ascontiguousarray(np.asarray(field, dtype=np.int8).ravel())
            fp = fa.ctypes.data_as(C.c_void_p)
        h = self.lib.orc_chain_new(kind, Lx, Ly, pbc, t, U, dtau, L, stab,
                                   seed, fp, delay, int(drift))
        ch = _Chain(self.lib, "orc_", h, n, L)
        ch.kind, ch.Lx, ch.Ly = kind, Lx, (Ly if kind == LAT_SQUARE else 1)
        ch.U = U
        return ch

    def model(self, ch):
        n = ch.n
        eK, eKi, th = np.zeros(n * n), np.zeros(n * n), np.zeros(n * n)
        bp = np.zeros(n, dtype=np.int32)
        consts = np.zeros(7)
        self.lib.orc_chain_model(ch.h, eK, eKi, th, bp, consts)
        return dict(expK=_fortran(eK, n), expKinv=_fortran(eKi, n),
                    thop=_fortran(th, n), bipart=bp, consts=consts)

    def drift(self, ch):
        out = np.zeros(3)
        self.lib.orc_chain_drift(ch.h, out)
        return out

    def measure(self, ch, sel=0):
        out = np.zeros(5)
        n = ch.n
        szz, sperp = np.zeros(n), np.zeros(n)
        nq = self.lib.orc_chain_measure(ch.h, out, sel, szz, sperp)
        return out, szz[:nq], sperp[:nq]

    def measure_g(self, thop, U, Gu, Gd):
        n = Gu.shape[0]
        out = np.zeros(5)
        self.lib.orc_measure_g(n, _cm(thop), U, _cm(Gu), _cm(Gd), out)
        return out

    def spin_g(self, Lx, Ly, sel, Gu, Gd):
        n = Gu.shape[0]
        szz, sperp = np.zeros(n), np.zeros(n)
        nq = self.lib.orc_spin_g(n, Lx, Ly, sel, _cm(Gu), _cm(Gd), szz, sperp)
        return szz[:nq], sperp[:nq]

    def udv_inv(self, U, D, T):
        n = U.shape[0]
        g = np.zeros(n * n)
        ds = C.c_int()
        rc = self.lib.orc_udv_inv(n, _cm(U), np.ascontiguousarray(D, dtype=np.float64),
                                  _cm(T), g, C.byref(ds))
        return rc, _fortran(g, n), ds.value

    def expm_sym(self, A, scale):
        n = A.shape[0]
        out = np.zeros(n * n)
        self.lib.orc_expm_sym(n, _cm(A), scale, out)
        return _fortran(out, n)

    def replica_seed(self, base, b, r):
        return self.lib.orc_replica_seed(base, b, r)

    def jackknife(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        m, e = C.c_double(), C.c_double()
        self.lib.orc_jackknife(x, len(x), C.byref(m), C.byref(e))
        return m.value, e.value

    def rng(self, seed, k):
        out = np.zeros(k)
        self.lib.orc_rng(seed, k, out)
        return out


def _cm(A):
    """numpy [i, j] -> contiguous column-major buffer."""
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T).ravel()


class Reference:
    """The unmodified reference engine (oracle/_ref/libdqmcref.so)."""

    PATH = os.path.join(HERE, "_ref", "libdqmcref.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self, path=None):
        lib = C.CDLL(path or self.PATH)
        lib.ref_chain_new.restype = C.c_void_p
        lib.ref_chain_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_double, C.c_double, C.c_double,
                                      C.c_int, C.c_int, C.c_ulonglong,
                                      C.c_void_p, C.c_int]
        lib.ref_chain_new_mode.restype = C.c_void_p
        lib.ref_chain_new_mode.argtypes = lib.ref_chain_new.argtypes + [C.c_int, C.c_int]
        lib.ref_chain_sweep.argtypes = [C.c_void_p, C.c_int]
        lib.ref_chain_state.argtypes = [C.c_void_p, _dp, _dp, _bp, _up,
                                        C.c_void_p, C.c_void_p, _up]
        lib.ref_chain_model.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip]
        lib.ref_chain_drift.argtypes = [C.c_void_p, _dp]
        lib.ref_chain_measure.argtypes = [C.c_void_p, _dp, C.c_char_p,
                                          C.c_void_p, C.c_void_p]
        lib.ref_green_scratch.argtypes = [C.c_void_p, C.c_int, _dp, C.c_void_p]
        lib.ref_wrap.argtypes = [C.c_void_p, C.c_int, _dp]
        lib.ref_chain_free.argtypes = [C.c_void_p]
        lib.ref_udv_inv.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, _dp,
                                    C.c_void_p]
        lib.ref_udv_recenter.argtypes = [C.c_int, _dp, C.c_void_p]
        lib.ref_expm_sym.argtypes = [C.c_int, _dp, C.c_double, _dp]
        lib.ref_replica_seed.restype = C.c_ulonglong
        lib.ref_replica_seed.argtypes = [C.c_ulonglong, C.c_int, C.c_int]
        lib.ref_jackknife.argtypes = [_dp, C.c_int, C.c_void_p, C.c_void_p]
        lib.ref_rng_first.restype = C.c_double
        lib.ref_rng_first.argtypes = [C.c_ulonglong, C.c_int, _dp]
        self.lib = lib

    def chain_mu(self, kind, Lx, Ly, U, dtau, L, stab, seed, half=True, mu=0.0,
                 two_spin=False, pbc=1, t=-1.0):
        """A reference chain on model_init(half, mu), optionally forced onto
        its two-spin path (ph_symmetric = 0)."""
        n = Lx * (Ly if kind == LAT_SQUARE else 1)
        self.lib.ref_chain_new_mu.restype = C.c_void_p
        self.lib.ref_chain_new_mu.argtypes = [C.c_int] * 4 + [C.c_double] * 3 + \
            [C.c_int, C.c_int, C.c_ulonglong, C.c_int, C.c_double, C.c_int]
        h = self.lib.ref_chain_new_mu(kind, Lx, Ly, pbc, t, U, dtau, L, stab, seed, int(half),
                                      mu, int(two_spin))
        ch = _Chain(self.lib, "ref_", h, n, L)
        ch.kind, ch.Lx, ch.Ly = kind, Lx, (Ly if kind == LAT_SQUARE else 1)
        return ch

    def chain(self, kind, Lx, Ly, U, dtau, L, stab, seed, field=None,
              pbc=1, t=-1.0, drift=False, alternating=False, rebuild=0):
        n = Lx * (Ly if kind == LAT_SQUARE else 1)
        fp = None
        if field is not None:
            fa = np.ascontiguousarray(np.asarray(field, dtype=np.int8).ravel())
            fp = fa.ctypes.data_as(C.c_void_p)
        h = self.lib.ref_chain_new_mode(kind, Lx, Ly, pbc, t, U, dtau, L, stab,
                                        seed, fp, int(drift), int(alternating), int(rebuild))
        ch = _Chain(self.lib, "ref_", h, n, L)
        ch.kind, ch.Lx, ch.Ly = kind, Lx, (Ly if kind == LAT_SQUARE else 1)
        return ch

    def model(self, ch):
        n = ch.n
        eK, eKi, th = np.zeros(n * n), np.zeros(n * n), np.zeros(n * n)
        bp = np.zeros(n, dtype=np.int32)
        self.lib.ref_chain_model(ch.h, eK, eKi, th, bp)
        return dict(expK=_fortran(eK, n), expKinv=_fortran(eKi, n),
                    thop=_fortran(th, n), bipart=bp)

    def drift(self, ch):
        out = np.zeros(5)
        self.lib.ref_chain_drift(ch.h, out)
        return out

    def measure(self, ch, selector=None):
        out = np.zeros(5)
        n = ch.n
        szz, sperp = np.zeros(n), np.zeros(n)
        if selector is None:
            self.lib.ref_chain_measure(ch.h, out, None, None, None)
            return out, None, None
        rc = self.lib.ref_chain_measure(ch.h, out, selector.encode(),
                                        szz.ctypes.data_as(C.c_void_p),
                                        sperp.ctypes.data_as(C.c_void_p))
        nq = 1 if selector == "af" else n
        assert rc == 0
        return out, szz[:nq], sperp[:nq]

    def udv_inv(self, U, D, T, log_offset=0.0):
        n = U.shape[0]
        g = np.zeros(n * n)
        ds = C.c_int()
        rc = self.lib.ref_udv_inv(n, _cm(U), np.ascontiguousarray(D, dtype=np.float64),
                                  _cm(T), log_offset, g, C.byref(ds))
        return rc, _fortran(g, n), ds.value

    def expm_sym(self, A, scale):
        n = A.shape[0]
        out = np.zeros(n * n)
        self.lib.ref_expm_sym(n, _cm(A), scale, out)
        return _fortran(out, n)

    def replica_seed(self, base, b, r):
        return self.lib.ref_replica_seed(base, b, r)

    def jackknife(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        m, e = C.c_double(), C.c_double()
        self.lib.ref_jackknife(x, len(x), C.byref(m), C.byref(e))
        return m.value, e.value

    def rng(self, seed, k):
        out = np.zeros(k)
        self.lib.ref_rng_first(seed, k, out)
        return out
