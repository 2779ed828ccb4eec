"""Flow/control parameters: ctypes mirror of ``ocfd_params`` (include/ocfd_ec_gpu.h).

``default_params`` restates set_default_parameter (sub_read_parameter.f90:30-106) and
``finalize`` restates set_const_para (sub_read_parameter.f90:371-429), so a caller can start
from raw namelist values (angles in degrees, Twall in kelvin) exactly like the Fortran driver.
"""
import ctypes
import math

PI = 3.1415926535897932  # const_var PI (sub_modules.f90:19)


class OcfdParams(ctypes.Structure):
    _fields_ = [
        ("nvar", ctypes.c_int),
        ("iflag_scheme", ctypes.c_int),
        ("bound_scheme", ctypes.c_int),
        ("iflag_flux", ctypes.c_int),
        ("iflag_reconstruction", ctypes.c_int),
        ("iflag_turbulence_model", ctypes.c_int),
        ("time_method", ctypes.c_int),
        ("if_viscous", ctypes.c_int),
        ("iflag_local_dt", ctypes.c_int),
        ("if_dtime_mesh", ctypes.c_int),
        ("iflag_limit_flow", ctypes.c_int),
        ("if_scheme_positivity", ctypes.c_int),
        ("cood_y_up", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("ma", ctypes.c_double),
        ("re", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("prl", ctypes.c_double),
        ("prt", ctypes.c_double),
        ("t_inf", ctypes.c_double),
        ("twall", ctypes.c_double),
        ("kt_inf", ctypes.c_double),
        ("wt_inf", ctypes.c_double),
        ("aoa", ctypes.c_double),
        ("aos", ctypes.c_double),
        ("a_alfa", ctypes.c_double),
        ("a_beta", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("dt_global", ctypes.c_double),
        ("dtmin", ctypes.c_double),
        ("dtmax", ctypes.c_double),
        ("w_lu", ctypes.c_double),
        ("mut_max", ctypes.c_double),
        ("p_outlet", ctypes.c_double),
        ("ldmin", ctypes.c_double),
        ("ldmax", ctypes.c_double),
        ("lpmin", ctypes.c_double),
        ("lpmax", ctypes.c_double),
        ("lumax", ctypes.c_double),
        ("lsamax", ctypes.c_double),
        ("ref_s", ctypes.c_double),
        ("ref_l", ctypes.c_double),
        ("centroid", ctypes.c_double * 3),
        ("cv", ctypes.c_double),
        ("cp", ctypes.c_double),
        ("res_inner_limit", ctypes.c_double),
        ("step_inner_limit", ctypes.c_int),
        ("if_residual_smoothing", ctypes.c_int),
    ]

    def copy(self):
        o = OcfdParams()
        ctypes.memmove(ctypes.byref(o), ctypes.byref(self), ctypes.sizeof(OcfdParams))
        return o

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name == "centroid" else v
        return d


def default_params(**raw):
    """set_default_parameter (sub_read_parameter.f90:30-106), then namelist overrides."""
    p = OcfdParams()
    p.ma, p.re, p.gamma = 1.0, 1000.0, 1.4
    p.aoa, p.aos = 0.0, 0.0
    p.p_outlet = -1.0
    p.iflag_turbulence_model = 0
    p.if_viscous = 1
    p.iflag_local_dt = 1
    p.dt_global = 0.01
    p.cfl = 1.0
    p.dtmax, p.dtmin = 10.0, 1.0e-9
    p.time_method = 0
    p.w_lu = 1.0
    p.if_dtime_mesh = 1
    p.iflag_scheme = 5
    p.iflag_flux = 5
    p.iflag_reconstruction = 0
    p.t_inf = 288.15
    p.twall = -1.0
    p.kt_inf, p.wt_inf = 1.0e-5, 0.01
    p.mut_max = -1.0
    p.bound_scheme = 4
    p.ref_s, p.ref_l = 1.0, 1.0
    p.centroid[0] = p.centroid[1] = p.centroid[2] = 0.0
    p.cood_y_up = 1
    p.iflag_limit_flow = 1
    p.prl, p.prt = 0.7, 0.9
    p.ldmin, p.ldmax, p.lpmin, p.lpmax, p.lumax, p.lsamax = 1.0e-6, 1000.0, 1.0e-6, 1000.0, 1000.0, 1000.0
    p.if_scheme_positivity = 1
    p.precision = 0
    p.step_inner_limit, p.res_inner_limit = 20, 1.0e-10
    for k, v in raw.items():
        if k == "centroid":
            for q in range(3):
                p.centroid[q] = v[q]
        else:
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
    return p


def finalize(p):
    """set_const_para (sub_read_parameter.f90:371-429), in place; returns p."""
    p.twall = p.twall / p.t_inf
    p.lpmin = p.lpmin / (p.gamma * p.ma * p.ma)
    p.lpmax = p.lpmax / (p.gamma * p.ma * p.ma)
    if p.bound_scheme == -1:
        p.bound_scheme = p.iflag_scheme
    if p.if_viscous == 0:
        p.iflag_turbulence_model = 0
    if p.iflag_turbulence_model in (2, 21):
        p.nvar = 6
    elif p.iflag_turbulence_model == 3:
        p.nvar = 7
    else:
        p.nvar = 5
    p.aoa = p.aoa * PI / 180.0
    p.aos = p.aos * PI / 180.0
    if p.cood_y_up == 1:
        p.a_alfa, p.a_beta = p.aoa, p.aos
    else:
        p.a_alfa, p.a_beta = p.aos, p.aoa
    p.cv = 1.0 / (p.gamma * (p.gamma - 1.0) * p.ma * p.ma)
    p.cp = p.cv * p.gamma
    return p


def make_params(**raw):
    """default_params(**raw) followed by finalize()."""
    return finalize(default_params(**raw))


def nvar_of(p):
    return int(p.nvar)
