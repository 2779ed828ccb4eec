"""Cases that drive the solver into its rarely taken, default-on branches.

Each case is a small mesh with flow parameters and a state prepared on the host (read back after
a few ordinary iterations, changed in a few cells, written back with set_state), the way a
restart from a damaged flow file or a diverging iteration would reach these branches:

* limit_flow_U (sub_limitflow.f90:24-176): cells outside the density / velocity bounds after the
  update are replaced by the average of their good neighbours (or clamped when none is good),
  and the block's IF_OverLimit flag is set for good;
* limit_flow_SA (sub_limitflow.f90:182-231): U6 below SAmin is clamped, U6 above LSAmax is
  replaced by the average of its neighbours in the serial loop order;
* what IF_OverLimit switches on: the UD1 scheme on every face (sub_Residual.f90:227-245), no
  viscous flux and Surf = 0 (734-750), dt x 0.1 (sub_time_acceleraction.f90:74-79);
* the positivity fallback (sub_Residual.f90:283-299): a reconstructed density or pressure at or
  below 1e-20 falls back to the cell values;
* limit_mut with MUT_MAX >= 0 (sub_Residual.f90:1387-1408).

The bounds are tightened through the parameters the reference reads from control.ec (Ldmin,
Ldmax, Lumax, LSAmax) so that mild, finite states cross them.  Every state here stays finite: the
limiter repairs a cell before the next residual reads it.
"""
from ocfd_b200 import cases

SST_INF = dict(kt_inf=1e-8, wt_inf=1e-5)
TIGHT = dict(ldmin=0.5, ldmax=2.0, lumax=3.0, lsamax=50.0)


def set_prim(U, i, j, k, gamma, rho=None, u=None, p=None):
    """Change density, x-velocity or pressure of cell (i,j,k) of a Fortran-layout state
    U[k+3, j+3, i+3, m], keeping the other primitive values."""
    c = U[k + 3, j + 3, i + 3]
    d = c[0]
    uu, vv, ww = c[1] / d, c[2] / d, c[3] / d
    pp = (c[4] - 0.5 * d * (uu * uu + vv * vv + ww * ww)) * (gamma - 1.0)
    d = d if rho is None else rho
    uu = uu if u is None else u
    pp = pp if p is None else p
    c[0], c[1], c[2], c[3] = d, d * uu, d * vv, d * ww
    c[4] = pp / (gamma - 1.0) + 0.5 * d * (uu * uu + vv * vv + ww * ww)


def _bad_cells(cells, sa=()):
    """A state change: cells (i, j, k, field, value) with field 'rho' or 'u', and SA cells
    (i, j, k, U6 value)."""
    def prep(U, gamma):
        for i, j, k, f, v in cells:
            set_prim(U, i, j, k, gamma, **{f: v})
        for i, j, k, v in sa:
            U[k + 3, j + 3, i + 3, 5] = v
    return prep


CLUSTER = [(i, j, k, "rho", 2.8 + 0.05 * (i + j + k)) for i in (9, 10, 11) for j in (4, 5, 6) for k in (1, 2, 3)]
CLUSTER_CENTRE = (10, 5, 2)


def limiter_cases():
    """name -> () -> (params, case, warm-up iterations, {block: prep(U, gamma)}, iterations)."""
    foil_cells = [(20, 6, 1, "rho", 2.6), (40, 8, 2, "u", 3.8), (30, 3, 1, "rho", 0.3)]
    return {
        # one block: density above and below the bounds, velocity above, U6 < 0 and U6 > LSAmax
        "foil_sa_lusgs": lambda: (*cases.airfoil(ni=65, nj=17, scheme=5, flux=4, turb=2, **TIGHT), 2,
                                  {0: _bad_cells(foil_cells, sa=[(10, 4, 1, -3.0), (50, 10, 2, 80.0), (51, 10, 2, 70.0)])}, 8),
        # WENO5 interior: under OverLimit every face of the block switches to UD1
        "foil_sa_weno5": lambda: (*cases.airfoil(ni=65, nj=17, scheme=7, flux=4, turb=2, **TIGHT), 2,
                                  {0: _bad_cells(foil_cells)}, 6),
        # eight blocks, bad cells in block 2 only: its flag is set, the others stay clear
        "wing8_sa": lambda: (*cases.config2_small(**TIGHT), 2,
                             {2: _bad_cells([(5, 8, 4, "rho", 2.7), (6, 9, 5, "u", 4.0)], sa=[(7, 10, 3, 75.0)])}, 6),
        # SST (NV = 7, no SA limiter), RK3: the limiter runs after every stage
        "foil_sst_rk3": lambda: (*cases.airfoil(ni=65, nj=17, scheme=5, flux=3, turb=3, time_method=3, cfl=1.0, **SST_INF,
                                                **TIGHT), 2, {0: _bad_cells(foil_cells)}, 5),
        # inviscid, LU-SGS: a 3 x 3 x 3 cluster of bad cells, so the centre cell has no good
        # neighbour and is clamped to the bounds instead of averaged
        "bump_euler": lambda: (*cases.config1(scale=0.25, **TIGHT), 2, {0: _bad_cells(CLUSTER)}, 5),
    }


POCKET_CELLS = ((10, 5, 2), (11, 5, 2))   # two cells along i at 1e-4 of the free-stream pressure


def positivity_case(scheme):
    """Channel bump (Euler) with a two-cell low-pressure pocket along i: the reconstruction of
    the pressure at the face between the two cells goes negative for UD3, UD5 and WENO5."""
    p, case = cases.config1(scale=0.25, iflag_scheme=scheme)
    pinf = 1.0 / (p.gamma * p.ma * p.ma)

    def prep(U, gamma):
        for i, j, k in POCKET_CELLS:
            set_prim(U, i, j, k, gamma, p=1e-4 * pinf)
    return p, case, 2, {0: prep}, 4


def mut_max_case(turb):
    """Airfoil with MUT_MAX >= 0: mu_t capped at MUT_MAX * mu (2 for SA; 0.005 for SST, whose
    eddy viscosity is small after the first iterations from free stream)."""
    if turb == 2:
        p, case = cases.airfoil(ni=65, nj=17, scheme=5, flux=4, turb=2, mut_max=2.0)
    else:
        p, case = cases.airfoil(ni=65, nj=17, scheme=5, flux=3, turb=3, mut_max=0.005, **SST_INF)
    return p, case, 20, {}, 6


def prepare(solver, params, warm, preps):
    """Advance the solver warm iterations, then apply the state changes block by block."""
    if warm:
        solver.advance(warm)
    for b, prep in preps.items():
        U = solver.get_state(b)
        prep(U, params.gamma)
        solver.set_state(b, U)
