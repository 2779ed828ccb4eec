"""Batches of independent solves in one handle (ocfd_create_batch): every solve of a batch gives
bit for bit the result it gives alone (same kernels, per-block arithmetic, per-solve reductions
in a fixed order), for uneven mesh sizes and different flow conditions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def items(precision=0):
    from ocfd_b200 import cases
    return [
        cases.airfoil(ni=65, nj=17, m=0.02, t=0.12, ma=0.7, aoa=2.0, precision=precision),
        cases.airfoil(ni=81, nj=25, m=0.0, t=0.10, ma=0.5, aoa=-1.0, precision=precision),
        cases.airfoil(ni=49, nj=21, m=0.04, t=0.15, ma=0.8, aoa=4.0, precision=precision),
    ]


def run(s, steps):
    s.advance(steps)
    return s


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_alone(gpu, precision):
    its = items(precision)
    batch = run(gpu.Batch(its), 6)
    rmax, rrms = batch.residual_all()
    ft, cl, cd, cs = batch.forces_all()
    for q, (p, case) in enumerate(its):
        alone = run(gpu.Solver(p, case), 6)
        am, ar = alone.residual()
        aft, acl, acd, acs = alone.forces()
        assert np.array_equal(ar, rrms[q]) and np.array_equal(am, rmax[q]), q
        assert np.array_equal(aft, ft[q]) and acl == cl[q] and acd == cd[q], q
        for b in range(len(case.dims)):
            assert np.array_equal(alone.get_state(b), batch.get_state(batch.blk0[q] + b)), (q, b)
        alone.close()
    batch.close()


def test_batch_matches_oracle(gpu, oracle):
    """Each solve of an FP64 batch against the oracle run of that case alone."""
    its = items(0)
    batch = run(gpu.Batch(its), 4)
    _, rrms = batch.residual_all()
    _, cl, cd, _ = batch.forces_all()
    for q, (p, case) in enumerate(its):
        o = oracle.OracleCase(p, case)
        o.advance(4)
        np.testing.assert_allclose(rrms[q][:6], o.residual()[1][:6], rtol=1e-11)
        _, ocl, ocd, _ = o.forces()
        assert abs(cl[q] - ocl) <= 1e-10 * abs(ocl) and abs(cd[q] - ocd) <= 1e-10 * abs(ocd)
        o.close()
    batch.close()


def test_footprint_bounds_allocation(gpu):
    import torch
    from ocfd_b200 import cases
    p, case = cases.config2_medium()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    s = gpu.Solver(p, case)
    s.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    used = free0 - free1
    est = gpu.footprint(p, case)
    assert used <= est <= 2 * used + (64 << 20), (used, est)
    s.close()


def test_config4_batch_runs(gpu):
    """The 64-airfoil batch (uneven 129x33 .. 385x97 O-meshes, SA, AUSMPW + MUSCL3, mixed) in
    one handle: one graph launch per step for all 64 solves, finite residuals and forces."""
    from ocfd_b200 import cases
    its = cases.config4_batch(n=64)
    b = gpu.Batch(its)
    assert b.nsolve == 64
    b.advance(20)
    _, rrms = b.residual_all()
    _, cl, cd, _ = b.forces_all()
    assert np.all(np.isfinite(rrms)) and np.all(np.isfinite(cl)) and np.all(np.isfinite(cd))
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_reset_solve_starts_over_like_a_new_handle(gpu, precision):
    """ocfd_reset_solve: a slot of a running batch takes a new case on its mesh (other Mach, AoA,
    Re); after it, that solve's states, norms and forces equal a new handle holding the case alone
    bit for bit, and the other solve is exactly where it would be without the reset."""
    from ocfd_b200 import cases
    a = cases.airfoil(ni=65, nj=17, ma=0.6, aoa=1.0, precision=precision)
    b = cases.airfoil(ni=81, nj=21, ma=0.7, aoa=2.5, m=0.03, precision=precision)
    c = cases.airfoil(ni=81, nj=21, ma=0.5, aoa=4.0, m=0.03, re=3.0e6, precision=precision)   # b's mesh
    assert all(np.array_equal(x, y) for x, y in zip(b[1].xyz, c[1].xyz))
    bt = gpu.Batch([a, b])
    bt.advance(30)
    bt.reset_solve(1, c[0])
    bt.advance(20)
    alone = gpu.Solver(*c)
    alone.advance(20)
    nb0 = len(a[1].dims)
    for k in range(alone.nblk):
        assert np.array_equal(bt.get_state(nb0 + k), alone.get_state(k))
    (mx, rm), (amx, arm) = bt.residual_all(), alone.residual()
    assert np.array_equal(rm[1], arm) and np.array_equal(mx[1], amx)
    ft, cl, cd, cs = bt.forces_all()
    _, acl, acd, _ = alone.forces()
    assert cl[1] == acl and cd[1] == acd
    ref = gpu.Batch([a, b])
    ref.advance(50)
    for k in range(nb0):
        assert np.array_equal(bt.get_state(k), ref.get_state(k))
    for s in (bt, alone, ref):
        s.close()


def test_reset_solve_with_a_wider_boundary_scheme(gpu):
    """A reset that changes a slot's boundary scheme to one whose stencil reaches deeper across a
    physical face (MUSCL2C, one ghost layer, to WENO7, three) recomputes the primitive region: the
    slot then equals a new handle with the case alone, bit for bit, and the other slot is untouched.
    A reset to a reconstruction the step was not built for is refused."""
    from ocfd_b200 import cases
    from ocfd_b200.capi import OcfdError
    a = cases.airfoil(ni=65, nj=17, ma=0.6, aoa=1.0)
    b = cases.airfoil(ni=81, nj=21, ma=0.7, aoa=2.5, m=0.03)
    c = cases.airfoil(ni=81, nj=21, ma=0.6, aoa=3.0, m=0.03, scheme=9, bound_scheme=9)   # b's mesh
    assert int(b[0].bound_scheme) == 4 and int(c[0].bound_scheme) == 9
    bt = gpu.Batch([a, b])
    bt.advance(10)
    bt.reset_solve(1, c[0])
    bt.advance(10)
    alone = gpu.Solver(*c)
    alone.advance(10)
    nb0 = len(a[1].dims)
    for k in range(alone.nblk):
        assert np.array_equal(bt.get_state(nb0 + k), alone.get_state(k))
    ref = gpu.Batch([a, b])
    ref.advance(20)
    for k in range(nb0):
        assert np.array_equal(bt.get_state(k), ref.get_state(k))
    d = cases.airfoil(ni=81, nj=21, ma=0.6, aoa=3.0, m=0.03, iflag_reconstruction=1)
    with pytest.raises(OcfdError):
        bt.reset_solve(1, d[0])
    for s in (bt, alone, ref):
        s.close()
