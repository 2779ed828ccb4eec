"""Residual smoothing and explicit Euler in the oracle against an independent numpy restatement.

* Residual_smoothing / tridiagonal (sub_time_acceleraction.f90:119-241): the oracle's smoothed
  residual equals the numpy line solves (i, then j, then k) applied to the unsmoothed residual of
  the same state, with the coefficients from the spectral radii (comput_Lijk, 7-56) and the
  normal Mach number restated in numpy; subsonic, supersonic (Mn > 1) and reversed (Mn < -1)
  lines, and lines of two cells (held unchanged) are covered.
* NS_Time_advance_1Euler (sub_time_advance.f90:217-260): after one step the interior is
  Un + dt Res/vol of the starting state, bit for bit.
"""
import numpy as np
import pytest

from meshes import wavy_box
from ocfd_b200.params import make_params


def _interior(o, b, name):
    """Cells 1..n-1 of an oracle cell array, whatever its lower bounds."""
    a, lo, hi = o.get_array(b, name)
    n = o.state_shape(b)                       # (nz+7, ny+7, nx+7, nv)
    cells = [n[2] - 8, n[1] - 8, n[0] - 8]     # interior cells per direction (i, j, k)
    sl = tuple(slice(1 - lo[d], 1 - lo[d] + cells[d]) for d in (2, 1, 0))
    return a[sl]


def _perturbed(o, seed=3):
    rng = np.random.default_rng(seed)
    for b in range(o.nblk):
        U = o.get_state(b)
        U[..., 0] *= 1.0 + 0.02 * rng.standard_normal(U.shape[:3])
        U[..., 1:4] += 0.05 * rng.standard_normal(U.shape[:3] + (3,)) * U[..., :1]
        o.set_state(b, U)


def _thomas(a, b, c, R):
    """tridiagonal along axis 0 with both end values held; a, b, c (n, ...), R (n, ..., 5)."""
    n = R.shape[0]
    Rs = R.copy()
    if n < 3:
        return Rs
    P = np.zeros(a.shape)
    Q = np.zeros(R.shape)
    Q[0] = R[0]
    for q in range(1, n - 1):
        tmp = 1.0 / (a[q] * P[q - 1] + b[q])
        P[q] = -c[q] * tmp
        Q[q] = (R[q] - a[q][..., None] * Q[q - 1]) * tmp[..., None]
    for q in range(n - 2, 0, -1):
        Rs[q] = P[q][..., None] * Rs[q + 1] + Q[q]
    return Rs


def _smooth_numpy(o, p, b, Res):
    """Residual_smoothing of block b on Res (nz-1, ny-1, nx-1, 5), interior cells."""
    U = o.get_state(b)[3:-3, 3:-3, 3:-3][1:-1, 1:-1, 1:-1]     # cells 1..n-1, (k, j, i, m)
    d = U[..., 0]
    u, v, w = U[..., 1] / d, U[..., 2] / d, U[..., 3] / d
    T = (U[..., 4] - 0.5 * d * (u * u + v * v + w * w)) / (p.cv * d)
    cc = np.sqrt(T) / p.ma
    Lc, nrm = [], []
    for dn, (S, n1, n2, n3) in enumerate((("Si", "ni1", "ni2", "ni3"), ("Sj", "nj1", "nj2", "nj3"), ("Sk", "nk1", "nk2", "nk3"))):
        arrs = [o.get_array(b, x)[0] for x in (S, n1, n2, n3)]      # faces 1..n, (k, j, i)

        def avg(a, dn=dn):
            lo = a[:-1, :-1, :-1]
            hi = [a[:-1, :-1, 1:], a[:-1, 1:, :-1], a[1:, :-1, :-1]][dn]
            return lo + hi
        sn = [avg(a) for a in arrs[1:]]
        un = 0.5 * (u * sn[0] + v * sn[1] + w * sn[2])
        Lc.append((np.abs(un) + cc) * (avg(arrs[0]) * 0.5))
        nrm.append(0.5 * (u * sn[0] + v * sn[1] + w * sn[2]) / cc)
    R = Res.copy()
    for dn in range(3):
        o1, o2 = [q for q in range(3) if q != dn]
        ei = np.minimum(np.minimum(1.0, Lc[dn] / Lc[o1]), Lc[dn] / Lc[o2])
        Mn = nrm[dn]
        a = np.where(Mn > 1.0, -ei, np.where(Mn < -1.0, 0.0, -ei))
        bb = np.where(Mn > 1.0, 1.0 + ei, np.where(Mn < -1.0, 1.0 + ei, 1.0 + 2.0 * ei))
        c = np.where(Mn > 1.0, 0.0, np.where(Mn < -1.0, -ei, -ei))
        ax = 2 - dn                                                  # (k, j, i) axis of direction dn
        mv = lambda x: np.moveaxis(x, ax, 0)
        R = np.moveaxis(_thomas(mv(a), mv(bb), mv(c), np.moveaxis(R, ax, 0)), 0, ax)
    return R, nrm[0]


@pytest.mark.parametrize("ma,aoa", [(0.5, 3.0), (1.6, 10.0), (1.6, 180.0)])
def test_smoothing_matches_numpy_restatement(oracle, ma, aoa):
    case = wavy_box(nx=13, ny=9, nz=3, cuts=(6,))          # nz = 3: k-lines of two cells, held
    runs = []
    for sm in (0, 1):
        p = make_params(ma=ma, aoa=aoa, iflag_scheme=5, iflag_flux=4, if_residual_smoothing=sm)
        o = oracle.OracleCase(p, case)
        _perturbed(o)
        o.compute_residual(False)
        runs.append((p, o, [_interior(o, b, "Res") for b in range(o.nblk)]))
    (p, o0, R0), (_, o1, R1) = runs
    for b in range(o0.nblk):
        assert np.abs(R1[b][..., :5] - R0[b][..., :5]).max() > 1e-6 * np.abs(R0[b][..., :5]).max()
        want, mn_i = _smooth_numpy(o0, p, b, R0[b][..., :5])
        if ma > 1.0:   # the upwind branches are the ones exercised
            assert (mn_i > 1.0).all() if aoa < 90.0 else (mn_i < -1.0).all()
        scale = np.abs(want).max(axis=(0, 1, 2))
        assert (np.abs(R1[b][..., :5] - want).max(axis=(0, 1, 2)) <= 1e-12 * scale).all()
    o0.close()
    o1.close()


def test_smoothing_keeps_uniform_residual_lines_and_freestream(oracle):
    """A freestream on the unperturbed mesh has Res = 0: smoothing keeps it 0."""
    case = wavy_box(nx=9, ny=7, nz=5)
    p = make_params(ma=0.5, aoa=3.0, iflag_scheme=5, iflag_flux=4, if_residual_smoothing=1)
    o = oracle.OracleCase(p, case)
    o.compute_residual(False)
    r = _interior(o, 0, "Res")[..., :5]
    assert np.abs(r).max() < 1e-12
    o.close()


def test_euler1_step_is_un_plus_dt_res(oracle):
    case = wavy_box(nx=11, ny=9, nz=5, cuts=(5,))
    p = make_params(ma=0.6, aoa=5.0, iflag_scheme=5, iflag_flux=4, time_method=1, cfl=0.5, iflag_limit_flow=0)
    o = oracle.OracleCase(p, case)
    _perturbed(o)
    U0 = [o.get_state(b) for b in range(o.nblk)]
    o.compute_residual(False)
    Res = [_interior(o, b, "Res") for b in range(o.nblk)]
    dt = [_interior(o, b, "dt") for b in range(o.nblk)]
    vol = [_interior(o, b, "vol") for b in range(o.nblk)]
    k, _ = o.advance(1)
    assert k == 1
    for b in range(o.nblk):
        U1 = o.get_state(b)[4:-4, 4:-4, 4:-4]
        du = Res[b] / vol[b][..., None]
        want = U0[b][4:-4, 4:-4, 4:-4] + dt[b][..., None] * du
        assert np.array_equal(U1, want)
    o.close()
