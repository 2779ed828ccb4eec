"""ctypes binding of libocfd_b200.so (C-ABI in include/ocfd_ec_gpu.h).

There is no CPU fallback: if the library is missing or fails to load, every call raises.
"""
import ctypes
import os

import numpy as np

from . import ROOT_DIR
from .params import OcfdParams

LIB_PATH = os.path.join(ROOT_DIR, "libocfd_b200.so")
_lib = None

OCFD_OK, OCFD_ERR_ARG, OCFD_ERR_CUDA, OCFD_ERR_OOM, OCFD_ERR_NAN, OCFD_ERR_TIMEOUT, OCFD_ERR_UNSUPPORTED = 0, -1, -2, -3, -4, -5, -6
OCFD_ERR_COMM = -8

EXPORTED = [
    "ocfd_default_params", "ocfd_finalize_params", "ocfd_create", "ocfd_destroy", "ocfd_last_error", "ocfd_state_size",
    "ocfd_set_state", "ocfd_get_state", "ocfd_init_flow", "ocfd_advance", "ocfd_residual", "ocfd_forces",
    "ocfd_limiter_status", "ocfd_array_shape", "ocfd_get_array", "ocfd_version", "ocfd_compute_residual",
    "ocfd_stream", "ocfd_profile", "ocfd_launches_per_step", "ocfd_create_batch", "ocfd_nsolve", "ocfd_reset_solve",
    "ocfd_residual_all", "ocfd_forces_all", "ocfd_footprint", "ocfd_synchronize", "ocfd_residual_static",
    "ocfd_lu_tile_width", "ocfd_lu_kernel_version", "ocfd_lu_one_launch", "ocfd_create_part", "ocfd_part_blocks", "ocfd_part_plan",
]


class OcfdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (code %d)" % (msg, code))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OcfdError(-7, "libocfd_b200.so not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp, cp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_char_p
        pp = ctypes.POINTER(OcfdParams)
        L.ocfd_default_params.argtypes = [pp]
        L.ocfd_finalize_params.argtypes = [pp]
        L.ocfd_create.argtypes = [pp, ctypes.c_int, ip, ctypes.POINTER(dp), ip, ip, ctypes.POINTER(dp), ctypes.POINTER(vp)]
        L.ocfd_destroy.argtypes = [vp]
        L.ocfd_last_error.argtypes = [vp]
        L.ocfd_last_error.restype = cp
        L.ocfd_state_size.argtypes = [vp, ctypes.c_int]
        L.ocfd_state_size.restype = ctypes.c_longlong
        L.ocfd_set_state.argtypes = [vp, ctypes.c_int, dp]
        L.ocfd_get_state.argtypes = [vp, ctypes.c_int, dp]
        L.ocfd_init_flow.argtypes = [vp]
        L.ocfd_compute_residual.argtypes = [vp, ctypes.c_int]
        L.ocfd_advance.argtypes = [vp, ctypes.c_int, ip, dp]
        L.ocfd_residual.argtypes = [vp, dp, dp]
        L.ocfd_forces.argtypes = [vp, dp, dp, dp, dp]
        L.ocfd_limiter_status.argtypes = [vp, ctypes.c_int, ip, ip]
        L.ocfd_array_shape.argtypes = [vp, ctypes.c_int, cp, ip, ip, ip]
        L.ocfd_get_array.argtypes = [vp, ctypes.c_int, cp, dp]
        L.ocfd_version.restype = cp
        L.ocfd_stream.argtypes = [vp]
        L.ocfd_stream.restype = vp
        L.ocfd_profile.argtypes = [vp, ctypes.c_int, dp]
        L.ocfd_launches_per_step.argtypes = [vp]
        L.ocfd_create_batch.argtypes = [pp, ctypes.c_int, ip, ip, ctypes.POINTER(dp), ip, ip, ctypes.POINTER(dp), ctypes.POINTER(vp)]
        L.ocfd_nsolve.argtypes = [vp]
        L.ocfd_reset_solve.argtypes = [vp, ctypes.c_int, vp]
        L.ocfd_residual_all.argtypes = [vp, dp, dp]
        L.ocfd_forces_all.argtypes = [vp, dp, dp, dp, dp]
        L.ocfd_footprint.argtypes = [pp, ctypes.c_int, ip]
        L.ocfd_footprint.restype = ctypes.c_longlong
        L.ocfd_synchronize.argtypes = [vp]
        L.ocfd_residual_static.argtypes = [vp, dp, dp]
        L.ocfd_lu_tile_width.argtypes = [vp]
        L.ocfd_lu_kernel_version.argtypes = [vp]
        L.ocfd_lu_one_launch.argtypes = [vp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def footprint(params, case):
    """Device bytes a handle for this case would take (upper estimate, no device call)."""
    nijk = np.array([v for d in case.dims for v in d], dtype=np.int32)
    return int(lib().ocfd_footprint(ctypes.byref(params), len(case.dims), _ip(nijk)))


class Solver:
    """One case resident on the current GPU, driven through the C-ABI."""

    def __init__(self, params, case, dw=None):
        self._create([(params, case)], dw)

    def _create(self, items, dw=None):
        L = lib()
        self.cases = [c for _, c in items]
        self.case = self.cases[0]
        self.params = items[0][0].copy()
        self.params_list = [p.copy() for p, _ in items]
        flats = [c.flat() for c in self.cases]
        nijk = np.concatenate([f[0] for f in flats]).astype(np.int32)
        xyz = [a for f in flats for a in f[1]]
        nsub = np.concatenate([f[2] for f in flats]).astype(np.int32)
        inc = np.concatenate([f[3] for f in flats]).astype(np.int32)
        nblk_s = np.array([len(f[1]) for f in flats], dtype=np.int32)
        self._keep = (nijk, xyz, nsub, inc, nblk_s)
        xyz_ptrs = (ctypes.POINTER(ctypes.c_double) * len(xyz))(*[_dp(a) for a in xyz])
        dwp = None
        if dw is not None:
            self._dw = [np.ascontiguousarray(d, dtype=np.float64) for d in dw]
            dwp = (ctypes.POINTER(ctypes.c_double) * len(dw))(*[_dp(a) for a in self._dw])
        h = ctypes.c_void_p()
        if len(items) == 1:
            rc = L.ocfd_create(ctypes.byref(self.params), len(xyz), _ip(nijk), xyz_ptrs, _ip(nsub), _ip(inc), dwp, ctypes.byref(h))
        else:
            parr = (OcfdParams * len(items))(*self.params_list)
            rc = L.ocfd_create_batch(parr, len(items), _ip(nblk_s), _ip(nijk), xyz_ptrs, _ip(nsub), _ip(inc), dwp, ctypes.byref(h))
        if rc != 0:
            raise OcfdError(rc, "ocfd_create failed")
        self.h = h
        self.nblk = len(xyz)
        self.nsolve = len(items)
        self.blk0 = np.concatenate([[0], np.cumsum(nblk_s)]).astype(int)
        self.dims = [d for c in self.cases for d in c.dims]
        self.nvar = int(self.params.nvar)

    def close(self):
        if getattr(self, "h", None):
            lib().ocfd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise OcfdError(rc, "%s: %s" % (what, lib().ocfd_last_error(self.h).decode()))

    def advance(self, n=1):
        ks, tt = ctypes.c_int(), ctypes.c_double()
        self._check(lib().ocfd_advance(self.h, n, ctypes.byref(ks), ctypes.byref(tt)), "advance")
        return ks.value, tt.value

    def init_flow(self):
        self._check(lib().ocfd_init_flow(self.h), "init_flow")

    def compute_residual(self, lusgs=False):
        self._check(lib().ocfd_compute_residual(self.h, int(lusgs)), "compute_residual")

    def residual(self):
        a, b = np.zeros(7), np.zeros(7)
        rc = lib().ocfd_residual(self.h, _dp(a), _dp(b))
        if rc == OCFD_ERR_NAN:
            raise FloatingPointError(lib().ocfd_last_error(self.h).decode())
        self._check(rc, "residual")
        return a, b

    def residual_static(self):
        """ocfd_residual without any allocation (static device scratch, see the header)."""
        a, b = np.zeros(7), np.zeros(7)
        rc = lib().ocfd_residual_static(self.h, _dp(a), _dp(b))
        if rc == OCFD_ERR_NAN:
            raise FloatingPointError(lib().ocfd_last_error(self.h).decode())
        self._check(rc, "residual_static")
        return a, b

    def forces(self):
        ft = np.zeros(9)
        cl, cd, cs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(lib().ocfd_forces(self.h, _dp(ft), ctypes.byref(cl), ctypes.byref(cd), ctypes.byref(cs)), "forces")
        return ft, cl.value, cd.value, cs.value

    def state_shape(self, b):
        if not 0 <= b < self.nblk:
            raise OcfdError(OCFD_ERR_ARG, "block %d out of range (%d blocks)" % (b, self.nblk))
        nx, ny, nz = self.dims[b]
        return (nz + 7, ny + 7, nx + 7, self.nvar)

    def get_state(self, b, out=None):
        U = out if out is not None else np.empty(self.state_shape(b))
        self._check(lib().ocfd_get_state(self.h, b, _dp(U)), "get_state")
        return U

    def set_state(self, b, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(lib().ocfd_set_state(self.h, b, _dp(U)), "set_state")

    def limiter_status(self, b):
        n, o = ctypes.c_int(), ctypes.c_int()
        self._check(lib().ocfd_limiter_status(self.h, b, ctypes.byref(n), ctypes.byref(o)), "limiter_status")
        return n.value, o.value

    def get_array(self, b, name):
        lo, hi, nv = (ctypes.c_int * 3)(), (ctypes.c_int * 3)(), ctypes.c_int()
        self._check(lib().ocfd_array_shape(self.h, b, name.encode(), lo, hi, ctypes.byref(nv)), "array_shape " + name)
        shape = tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))
        if nv.value > 1:
            shape = shape + (nv.value,)
        out = np.empty(shape)
        self._check(lib().ocfd_get_array(self.h, b, name.encode(), _dp(out)), "get_array " + name)
        return out, tuple(lo), tuple(hi)


    def stream(self):
        """cudaStream_t (int) all of this handle's work is queued on."""
        return lib().ocfd_stream(self.h)

    PHASES = ("residual", "lusgs_lower", "lusgs_upper", "update_limit", "bc_halo", "step")

    def profile(self, nsteps=3):
        """Per-phase device ms accumulated over nsteps steps (dict)."""
        ms = np.zeros(8)
        self._check(lib().ocfd_profile(self.h, nsteps, _dp(ms)), "profile")
        return dict(zip(self.PHASES, ms[:6].tolist()))

    def launches_per_step(self):
        return int(lib().ocfd_launches_per_step(self.h))

    def lu_tile_width(self):
        """Columns per CTA tile of the LU-SGS sweeps, as picked by the creation-time autotuner."""
        return int(lib().ocfd_lu_tile_width(self.h))

    def lu_kernel_version(self):
        """LU-SGS wavefront kernel version in use (3 or 4; 2 with OCFD_LU_V2), as picked at creation."""
        return int(lib().ocfd_lu_kernel_version(self.h))

    def lu_one_launch(self):
        """True when both LU-SGS sweeps run as one launch (profile() then reports them as the lower one)."""
        return bool(lib().ocfd_lu_one_launch(self.h))

    def synchronize(self):
        self._check(lib().ocfd_synchronize(self.h), "synchronize")

    def residual_all(self):
        """(res_max, res_rms), each (nsolve, 7); NaN in a solve shows as NaN in its rms."""
        a, b = np.zeros(7 * self.nsolve), np.zeros(7 * self.nsolve)
        rc = lib().ocfd_residual_all(self.h, _dp(a), _dp(b))
        if rc not in (0, OCFD_ERR_NAN):
            self._check(rc, "residual_all")
        return a.reshape(self.nsolve, 7), b.reshape(self.nsolve, 7)

    def forces_all(self):
        """(ft (nsolve, 9), cl, cd, cs (nsolve,))."""
        n = self.nsolve
        ft, cl, cd, cs = np.zeros(9 * n), np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(lib().ocfd_forces_all(self.h, _dp(ft), _dp(cl), _dp(cd), _dp(cs)), "forces_all")
        return ft.reshape(n, 9), cl, cd, cs


class Batch(Solver):
    """Many independent cases in one handle: each step is one launch sequence over all blocks.
    items: list of (params, case).  Blocks are numbered globally in item order; solve q owns
    blocks blk0[q] .. blk0[q+1]-1."""

    def __init__(self, items, dw=None):
        self._create(list(items), dw)

    def reset_solve(self, q, params):
        """Solve q starts over with new parameters on its own mesh (ocfd_reset_solve)."""
        self._check(lib().ocfd_reset_solve(self.h, int(q), ctypes.byref(params)), "reset_solve")


def version():
    return lib().ocfd_version().decode()
