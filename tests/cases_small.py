"""Small parity cases: every scheme, flux, turbulence model and time method the hot path has,
on meshes the CPU oracle advances in well under a second per step."""
from ocfd_b200 import cases

SST_INF = dict(kt_inf=1e-8, wt_inf=1e-5)   # CFL3D-nondimensional k, omega far-field values


def small_cases():
    return {
        "bump1": lambda: cases.config1(scale=0.25),
        "bump2": lambda: cases.config1(scale=0.25, cuts_i=(12,)),
        "foil_sa_weno5_roe": lambda: cases.airfoil(ni=65, nj=17, scheme=7, flux=4),
        "foil_sa_muscl3_ausmpw": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=6),
        "foil_lam_rk3_hllc": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=3, turb=0, time_method=3, cfl=1.0),
        "foil_sst_lusgs_hllc": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=3, turb=3, **SST_INF),
        "foil_sst_rk3_hllc": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=3, turb=3, time_method=3, cfl=1.5, **SST_INF),
        "foil_sa_muscl2c_vl": lambda: cases.airfoil(ni=65, nj=17, scheme=4, flux=5, turb=2),
        "foil_sa_weno7_sw": lambda: cases.airfoil(ni=65, nj=17, scheme=9, flux=1, turb=2),
        "foil_sa_char_hll": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=2, turb=2, iflag_reconstruction=2),
        "foil_sa_cons_omuscl2_roe": lambda: cases.airfoil(ni=65, nj=17, scheme=6, flux=4, turb=2, iflag_reconstruction=1),
        "wing8": lambda: cases.config2_small(),
        "wing24_sst_roe": lambda: cases.config3_small(),
        "wing24_sst_rk3": lambda: cases.config3_small(time_method=3, cfl=0.5),
        "foil_sa_dual": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=4, turb=2, time_method=-1, dt_global=0.05,
                                              step_inner_limit=4, res_inner_limit=1e-14),
        "bump_dual": lambda: cases.config1(scale=0.25, time_method=-1, dt_global=0.2, step_inner_limit=3, res_inner_limit=1e-14),
        "bump_euler1": lambda: cases.config1(scale=0.25, cuts_i=(12,), time_method=1, cfl=0.5),
        "bump_euler1_smooth": lambda: cases.config1(scale=0.25, time_method=1, cfl=1.0, if_residual_smoothing=1),
        "foil_sa_lusgs_smooth": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=4, turb=2, if_residual_smoothing=1),
        "foil_lam_rk3_smooth": lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=4, turb=0, time_method=3, cfl=1.5,
                                                     if_residual_smoothing=1),
        # the schemes no other case uses as the interior scheme (sub_scheme.f90:6-96): UD1, NND2,
        # UD3, MUSCL2U, UD5, and UD1 as the boundary scheme
        "foil_sa_ud1_roe": lambda: cases.airfoil(ni=65, nj=17, scheme=0, flux=4, turb=2),
        "foil_lam_nnd2_vl": lambda: cases.airfoil(ni=65, nj=17, scheme=1, flux=5, turb=0),
        "bump_ud3_roe": lambda: cases.config1(scale=0.25, iflag_scheme=2),
        "foil_sa_muscl2u_sw": lambda: cases.airfoil(ni=65, nj=17, scheme=3, flux=1, turb=2),
        "bump_ud5_ausmpw": lambda: cases.config1(scale=0.25, iflag_scheme=8, iflag_flux=6),
        "foil_sa_ud3_bound_ud1": lambda: cases.airfoil(ni=65, nj=17, scheme=2, flux=4, turb=2, bound_scheme=0),
        # the wide boundary schemes, whose stencils at a physical face reach 2 (WENO5, UD5) and 3
        # (WENO7) ghost layers: the primitives are computed on exactly those layers there
        "foil_sa_weno7_bound_weno7": lambda: cases.airfoil(ni=65, nj=17, scheme=9, flux=4, turb=2, bound_scheme=9),
        "bump_weno5_bound_weno5": lambda: cases.config1(scale=0.25, cuts_i=(12,), iflag_scheme=7, bound_scheme=7),
        "foil_lam_ud5_bound_ud5": lambda: cases.airfoil(ni=65, nj=17, scheme=8, flux=6, turb=0, bound_scheme=8),
        "bump_dual_smooth": lambda: cases.config1(scale=0.25, cuts_i=(12,), time_method=-1, dt_global=0.2, step_inner_limit=3,
                                                  res_inner_limit=1e-14, if_residual_smoothing=1),
    }


# the subset whose golden fixtures are committed (tests/golden/)
GOLDEN_CASES = ("bump2", "foil_sa_weno5_roe", "foil_lam_rk3_hllc", "foil_sst_lusgs_hllc", "wing8")
GOLDEN_STEPS = 5
