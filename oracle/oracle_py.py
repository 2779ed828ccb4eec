"""ctypes binding of the CPU oracle (oracle/liboracle_ocfd.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, never by the product package.  The entry points mirror the product C-ABI
(include/ocfd_ec_gpu.h) with an ``oracle_`` prefix so parity tests read the same on both sides.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_ocfd.so")
_lib = None


def build(force=False):
    """Compile the oracle with its Makefile (g++ -O2 -ffp-contract=off)."""
    src = os.path.join(HERE, "ocfd_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle_ocfd.so"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp, cp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_char_p
        L.oracle_create.argtypes = [vp, ctypes.c_int, ip, ctypes.POINTER(dp), ip, ip, ctypes.POINTER(dp), ctypes.POINTER(vp)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_last_error.argtypes = [vp]
        L.oracle_last_error.restype = cp
        L.oracle_advance.argtypes = [vp, ctypes.c_int, ip, dp]
        L.oracle_init_flow.argtypes = [vp]
        L.oracle_compute_residual.argtypes = [vp, ctypes.c_int]
        L.oracle_residual.argtypes = [vp, dp, dp]
        L.oracle_forces.argtypes = [vp, dp, dp, dp, dp]
        L.oracle_state_size.argtypes = [vp, ctypes.c_int]
        L.oracle_state_size.restype = ctypes.c_longlong
        L.oracle_get_state.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_set_state.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_limiter_status.argtypes = [vp, ctypes.c_int, ip, ip]
        L.oracle_array_shape.argtypes = [vp, ctypes.c_int, cp, ip, ip, ip]
        L.oracle_get_array.argtypes = [vp, ctypes.c_int, cp, dp]
        L.oracle_flux_1d.argtypes = [dp, dp, dp, ctypes.c_double, ctypes.c_int]
        L.oracle_scheme.argtypes = [dp, ctypes.c_int, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class OracleCase:
    """One case on the CPU oracle; same methods as ocfd_b200.capi.Solver."""

    def __init__(self, params, case, dw=None):
        L = lib()
        self.case = case
        self.params = params
        nijk, xyz, nsub, inc = case.flat()
        self._keep = (nijk, xyz, nsub, inc)
        xyz_ptrs = (ctypes.POINTER(ctypes.c_double) * len(xyz))(*[_dp(a) for a in xyz])
        dwp = None
        if dw is not None:
            self._dw = [np.ascontiguousarray(d, dtype=np.float64) for d in dw]
            dwp = (ctypes.POINTER(ctypes.c_double) * len(dw))(*[_dp(a) for a in self._dw])
        h = ctypes.c_void_p()
        rc = L.oracle_create(ctypes.byref(params), len(xyz), _ip(nijk), xyz_ptrs, _ip(nsub), _ip(inc), dwp, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError("oracle_create failed: %d" % rc)
        self.h = h
        self.nblk = len(xyz)
        self.nvar = int(params.nvar)

    def close(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s failed (%d): %s" % (what, rc, lib().oracle_last_error(self.h).decode()))

    def advance(self, n=1):
        ks, tt = ctypes.c_int(), ctypes.c_double()
        self._check(lib().oracle_advance(self.h, n, ctypes.byref(ks), ctypes.byref(tt)), "advance")
        return ks.value, tt.value

    def init_flow(self):
        self._check(lib().oracle_init_flow(self.h), "init_flow")

    def compute_residual(self, lusgs=False):
        self._check(lib().oracle_compute_residual(self.h, int(lusgs)), "compute_residual")

    def residual(self):
        a, b = np.zeros(7), np.zeros(7)
        rc = lib().oracle_residual(self.h, _dp(a), _dp(b))
        if rc != 0:
            raise FloatingPointError(lib().oracle_last_error(self.h).decode())
        return a, b

    def forces(self):
        ft = np.zeros(9)
        cl, cd, cs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(lib().oracle_forces(self.h, _dp(ft), ctypes.byref(cl), ctypes.byref(cd), ctypes.byref(cs)), "forces")
        return ft, cl.value, cd.value, cs.value

    def state_shape(self, b):
        nx, ny, nz = self.case.dims[b]
        return (nz + 7, ny + 7, nx + 7, self.nvar)

    def get_state(self, b):
        U = np.empty(self.state_shape(b))
        self._check(lib().oracle_get_state(self.h, b, _dp(U)), "get_state")
        return U

    def set_state(self, b, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(lib().oracle_set_state(self.h, b, _dp(U)), "set_state")

    def limiter_status(self, b):
        n, o = ctypes.c_int(), ctypes.c_int()
        lib().oracle_limiter_status(self.h, b, ctypes.byref(n), ctypes.byref(o))
        return n.value, o.value

    def get_array(self, b, name):
        lo, hi, nv = (ctypes.c_int * 3)(), (ctypes.c_int * 3)(), ctypes.c_int()
        self._check(lib().oracle_array_shape(self.h, b, name.encode(), lo, hi, ctypes.byref(nv)), "array_shape " + name)
        shape = tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))
        if nv.value > 1:
            shape = shape + (nv.value,)
        out = np.empty(shape)
        self._check(lib().oracle_get_array(self.h, b, name.encode(), _dp(out)), "get_array " + name)
        return out, tuple(lo), tuple(hi)


def set_threads(n):
    """Host threads of the oracle's loop pool; returns the count in use."""
    return int(lib().oracle_set_threads(int(n)))


def threads():
    return int(lib().oracle_threads())


def flux_1d(QL, QR, gamma, iflux):
    F = np.zeros(5)
    QL = np.ascontiguousarray(QL, dtype=np.float64)
    QR = np.ascontiguousarray(QR, dtype=np.float64)
    lib().oracle_flux_1d(_dp(QL), _dp(QR), _dp(F), gamma, iflux)
    return F


def scheme(u8, s):
    u8 = np.ascontiguousarray(u8, dtype=np.float64)
    a, b = ctypes.c_double(), ctypes.c_double()
    lib().oracle_scheme(_dp(u8), s, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value
