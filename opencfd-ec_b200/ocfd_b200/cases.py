"""Benchmark and parity cases: mesh + flow parameters for each configuration.

config1: plain FP64 Euler channel bump, 129x65x17, MUSCL3 (van Albada) + Roe, LU-SGS CFL 5, M 0.5.
config2: plain FP64 RANS-SA swept wing, 8 uneven blocks, ~2.1M cells, WENO5 + Roe, LU-SGS,
         M 0.8, AoA 3 deg, Re 1e7 per chord.
config4: 2-D-extruded NACA 4-digit O-mesh airfoils (k = 3 nodes), SA, AUSMPW + MUSCL3, mixed.
Small variants of each are the parity cases (sizes the CPU oracle finishes in seconds).
"""
import numpy as np

from . import meshgen
from .params import make_params


def config1(scale=1.0, cuts_i=(), **over):
    ni = int(round((129 - 1) * scale)) + 1
    nj = int(round((65 - 1) * scale)) + 1
    nk = max(3, int(round((17 - 1) * scale)) + 1)
    case = meshgen.channel_bump(ni, nj, nk, cuts_i=cuts_i, name="config1_bump_%dx%dx%d" % (ni, nj, nk))
    raw = dict(ma=0.5, aoa=0.0, if_viscous=0, iflag_scheme=5, iflag_flux=4, time_method=0, cfl=5.0, t_end=1.0e9)
    raw.update(over)
    raw.pop("t_end")
    return make_params(**raw), case


def config2(ni=257, nj=97, nk_wing=61, nk_tip=26, i_cut=49, **over):
    case = meshgen.swept_wing(ni=ni, nj=nj, nk_wing=nk_wing, nk_tip=nk_tip, i_cut=i_cut,
                              name="config2_wing_%dx%dx%d" % (ni, nj, nk_wing + nk_tip - 1))
    raw = dict(ma=0.8, aoa=3.0, re=1.0e7, if_viscous=1, iflag_turbulence_model=2, iflag_scheme=7, iflag_flux=4,
               time_method=0, cfl=5.0, ref_s=meshgen.wing_ref_area(), ref_l=1.0)
    raw.update(over)
    return make_params(**raw), case


FUSELAGE = dict(length=4.0, fineness=8.0, xc=0.5)   # ellipsoid: 4 root chords long, fineness 8, centred at mid-chord


def config3(ni=449, nj=129, nk_wing=97, nk_tip=41, i_cut=86, j_cuts=(33, 73), **over):
    """Config 3: the swept wing with an ellipsoidal fuselage (length 4 chords, fineness 8) at its
    root, ~7.8 M cells in 24 uneven blocks (4 around the section x 3 wall-normal x 2 spanwise),
    RANS-SST, MUSCL3, LU-SGS, M 0.75, AoA 2 deg, Re 3e6, mixed precision by default (the FP64 run
    of the same case is precision=0).  The fuselage is the root surface lifted onto the half
    ellipsoid (meshgen.swept_wing); it keeps the root plane's symmetry condition, so it is a slip
    surface and its pressure is not in the integrated forces.

    The flux defaults to Roe, a stand-in: with HLLC as the configuration states (iflag_flux=3),
    the reference algorithm diverges in the first iterations on this wing-body, in the CPU
    restatement as on the GPU (its right star state carries v into the w-momentum,
    sub_flux_split.f90:67); config3_as_specified() builds that case.  LU-SGS runs at CFL 1.  The
    RK3 variant (time_method=3) of the configuration is at CFL 1.5, where explicit RK3 with the SST
    model diverges at the first step in the far field beyond the tip (at CFL 0.8 too; Euler,
    laminar and SA run); the stand-in uses CFL 0.5."""
    case = meshgen.swept_wing(ni=ni, nj=nj, nk_wing=nk_wing, nk_tip=nk_tip, i_cut=i_cut, j_cuts=j_cuts, fuselage=FUSELAGE,
                              name="config3_wingbody_%dx%dx%d_24blk" % (ni, nj, nk_wing + nk_tip - 1))
    raw = dict(ma=0.75, aoa=2.0, re=3.0e6, if_viscous=1, iflag_turbulence_model=3, iflag_scheme=5, iflag_flux=4,
               time_method=0, cfl=1.0, precision=1, kt_inf=1e-8, wt_inf=1e-5, ref_s=meshgen.wing_ref_area(), ref_l=1.0)
    raw.update(over)
    return make_params(**raw), case


def config3_as_specified(rk3=False, **over):
    """Config 3 exactly as stated: HLLC + MUSCL3, LU-SGS, or the RK3 variant at CFL 1.5."""
    if rk3:
        return config3(iflag_flux=3, time_method=3, cfl=1.5, **over)
    return config3(iflag_flux=3, **over)


def config3_small(**over):
    """A reduced config 3 (24 blocks) for oracle parity."""
    return config3(ni=41, nj=21, nk_wing=9, nk_tip=6, i_cut=9, j_cuts=(6, 12), precision=0, **over)


def config2_medium(**over):
    """The swept wing at a quarter of the cells (~0.5 M, ~0.6 GB on the device): larger than L2,
    small enough for multi-pass profiler captures."""
    return config2(ni=129, nj=97, nk_wing=31, nk_tip=14, i_cut=25, **over)


def config2_small(**over):
    """A reduced swept wing (8 blocks) for oracle parity."""
    return config2(ni=41, nj=17, nk_wing=9, nk_tip=6, i_cut=9, **over)


def airfoil(ni=129, nj=33, m=0.02, p=0.4, t=0.12, ma=0.7, aoa=2.0, re=6.0e6, scheme=5, flux=6, turb=2, precision=0,
            time_method=0, cfl=5.0, ds=2e-6, **over):
    case = meshgen.airfoil_omesh(ni=ni, nj=nj, nk=3, m=m, p=p, t=t, ds=ds, name="naca_%dx%d" % (ni, nj))
    raw = dict(ma=ma, aoa=aoa, re=re, if_viscous=1, iflag_turbulence_model=turb, iflag_scheme=scheme, iflag_flux=flux,
               time_method=time_method, cfl=cfl, precision=precision, ref_s=case.xyz[0][2].max() - case.xyz[0][2].min())
    raw.update(over)
    return make_params(**raw), case


def config4_batch(n=64, seed=1234, **over):
    """64 airfoil solves: O-mesh sizes uniform in 129x33 .. 385x97 (odd ni), NACA 4-digit camber
    U[0,0.04], thickness U[0.09,0.15], Mach U[0.3,0.85], AoA U[-2,6] deg, Re 6e6, SA, AUSMPW +
    MUSCL3, mixed precision.  Returns a list of (params, case)."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        ni = int(rng.integers(64, 193)) * 2 + 1      # 129..385, odd
        nj = int(rng.integers(33, 98))
        m = float(rng.uniform(0.0, 0.04))
        p = 0.4
        t = float(rng.uniform(0.09, 0.15))
        ma = float(rng.uniform(0.3, 0.85))
        aoa = float(rng.uniform(-2.0, 6.0))
        raw = dict(precision=1)
        raw.update(over)
        out.append(airfoil(ni=ni, nj=nj, m=m, p=p, t=t, ma=ma, aoa=aoa, re=6.0e6, scheme=5, flux=6, turb=2, **raw))
    return out
