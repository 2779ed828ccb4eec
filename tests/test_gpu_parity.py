"""CUDA path (through the C-ABI) against the CPU oracle on the same inputs.

FP64 path: geometry bit-for-bit up to 1e-13 relative (the mesh-metric formulas are evaluated in
the same order, FMA off), residual norms per step within 1e-11 relative (summation order of
the norms differs), forces within 1e-10, state within 1e-11 of its scale.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from cases_small import GOLDEN_CASES, GOLDEN_STEPS, small_cases

pytestmark = pytest.mark.gpu

GEOMETRY = ("vol", "Si", "Sj", "Sk", "ni1", "nk3", "ix1", "jy2", "kz3", "ix0", "dtime_mesh", "dw")
STEPS = 6


def overlap(a, lo, b, lo2):
    """Crop oracle array a (lower bounds lo) to GPU array b's extent (lower bounds lo2)."""
    if a.shape == b.shape:
        return a
    sl = tuple(slice(lo2[d] - lo[d], lo2[d] - lo[d] + b.shape[2 - d]) for d in (2, 1, 0))
    return a[sl]


def compare_geometry(o, g, names=GEOMETRY, rtol=1e-13):
    for b in range(o.nblk):
        for n in names:
            a, lo, _ = o.get_array(b, n)
            c, lo2, _ = g.get_array(b, n)
            a = overlap(a, lo, c, lo2)
            scale = max(np.abs(a).max(), 1e-300)
            err = np.abs(a - c).max() / scale
            assert err <= rtol, "block %d %s: %.3e" % (b, n, err)


def state_err(o, g):
    worst = 0.0
    for b in range(o.nblk):
        A, B = o.get_state(b), g.get_state(b)
        scale = np.maximum(np.abs(A).max(axis=(0, 1, 2)), 1e-30)
        worst = max(worst, float((np.abs(A - B).max(axis=(0, 1, 2)) / scale).max()))
    return worst


@pytest.mark.parametrize("name", list(small_cases()))
def test_parity_small_cases(gpu, oracle, name):
    p, case = small_cases()[name]()
    o = oracle.OracleCase(p, case)
    g = gpu.Solver(p, case)
    compare_geometry(o, g)
    assert state_err(o, g) == 0.0
    for it in range(STEPS):
        ko, to = o.advance(1)
        kg, tg = g.advance(1)
        assert ko == kg
        mo, ro = o.residual()
        mg, rg = g.residual()
        nv = p.nvar
        np.testing.assert_allclose(rg[:nv], ro[:nv], rtol=1e-11, err_msg="rms step %d" % it)
        np.testing.assert_allclose(mg[:nv], mo[:nv], rtol=1e-10, err_msg="max step %d" % it)
    fo, fg = o.forces(), g.forces()
    np.testing.assert_allclose(fg[0], fo[0], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(fg[1:], fo[1:], rtol=1e-10, atol=1e-14)
    assert state_err(o, g) <= 1e-11
    for b in range(o.nblk):
        assert g.limiter_status(b) == o.limiter_status(b)
    g.close()
    o.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_matches_golden_fixtures(gpu, name):
    """The committed fixtures (oracle output) reproduced by the CUDA path."""
    from golden.make_golden import interior_checksums
    gd = np.load(os.path.join(GOLDEN, "case_%s.npz" % name))
    p, case = small_cases()[name]()
    g = gpu.Solver(p, case)
    rms, rmax = [], []
    for _ in range(GOLDEN_STEPS):
        g.advance(1)
        a, b = g.residual()
        rmax.append(a)
        rms.append(b)
    np.testing.assert_allclose(np.array(rms), gd["res_rms"], rtol=1e-11, atol=1e-300)
    np.testing.assert_allclose(np.array(rmax), gd["res_max"], rtol=1e-10, atol=1e-300)
    ft, cl, cd, cs = g.forces()
    np.testing.assert_allclose([cl, cd, cs], gd["clcdcs"], rtol=1e-10, atol=1e-14)
    chk = np.stack([interior_checksums(g.get_state(b), case.dims[b]) for b in range(g.nblk)])
    np.testing.assert_allclose(chk, gd["state_checksums"], rtol=1e-11, atol=1e-13)
    g.close()


def test_residual_only_matches_oracle(gpu, oracle):
    """ocfd_compute_residual (no update) on the SA wing: Res, Lc, Lv, dt arrays."""
    from ocfd_b200 import cases
    p, case = cases.config2_small()
    o, g = oracle.OracleCase(p, case), gpu.Solver(p, case)
    o.advance(2)
    g.advance(2)
    o.compute_residual(False)
    g.compute_residual(False)
    for b in range(o.nblk):
        a, lo, _ = o.get_array(b, "Res")
        c, lo2, _ = g.get_array(b, "Res")
        a = overlap(a, lo, c, lo2)      # interior cells 1..n-1
        scale = np.maximum(np.abs(a).max(axis=(0, 1, 2)), 1e-300)
        assert (np.abs(a - c).max(axis=(0, 1, 2)) / scale).max() <= 1e-11
    g.close()
    o.close()


@pytest.mark.parametrize("name", ["foil_sa_muscl3_ausmpw", "wing8", "bump1"])
def test_mixed_precision_close_to_fp64(gpu, oracle, name):
    """Mixed path (FP32 primitives/metrics/fluxes, FP64 state, diagonal, norms, forces) stays
    close to the FP64 oracle after 10 steps: residual norms within 1e-3 of the largest component,
    CL/CD within 1e-4 of max(|C|, 0.01) (forces integrate O(1) pressures held in FP32)."""
    p, case = small_cases()[name]()
    q = p.copy()
    q.precision = 1
    o, g = oracle.OracleCase(p, case), gpu.Solver(q, case)
    for _ in range(10):
        o.advance(1)
        g.advance(1)
    ro, rg = o.residual()[1][:p.nvar], g.residual()[1][:p.nvar]
    assert np.all(np.abs(rg - ro) <= 1e-3 * np.abs(ro).max()), (ro, rg)
    fo, fg = o.forces(), g.forces()
    assert abs(fg[1] - fo[1]) <= 1e-4 * max(abs(fo[1]), 1e-2)
    assert abs(fg[2] - fo[2]) <= 1e-4 * max(abs(fo[2]), 1e-2)
    assert state_err(o, g) <= 1e-4
    g.close()
    o.close()


@pytest.mark.parametrize("turb,scheme", [(0, 7), (2, 5)])
def test_ragged_blocks_down_to_one_cell(gpu, oracle, turb, scheme):
    """Uneven blocks down to a single cell layer (a block of 2 nodes in i) and a 2-cell block, no
    wall (wall distance 1e8 everywhere): the interface copies of blocks thinner than LAP read
    ghost cells that other copies write, and the GPU orders them as the reference's
    subface-by-subface loop does (WENO5 reads all LAP ghost layers); the wavefront tiles, BC
    rounds and norms handle the thin blocks as the oracle does."""
    from meshes import wavy_box
    from ocfd_b200.params import make_params
    case = wavy_box(nx=21, ny=11, nz=7, cuts=(2, 4, 15))       # blocks of 1, 2, 11, 6 cells in i
    assert [d[0] - 1 for d in case.dims] == [1, 2, 11, 6]
    p = make_params(ma=0.5, aoa=3.0, if_viscous=int(turb > 0), iflag_turbulence_model=turb, iflag_scheme=scheme, iflag_flux=4,
                    re=1e5, cfl=2.0)
    o, g = oracle.OracleCase(p, case), gpu.Solver(p, case)
    for _ in range(4):
        o.advance(1)
        g.advance(1)
        np.testing.assert_allclose(g.residual()[1][:p.nvar], o.residual()[1][:p.nvar], rtol=1e-11, atol=1e-300)
    assert state_err(o, g) <= 1e-11
    g.close()
    o.close()
