"""The benchmark workloads at full size on the CUDA path.

Parity with the oracle where the oracle finishes in seconds (config 1 full, config 2 one step),
and size-independent properties elsewhere: schedule invariance of the LU-SGS sweep (pipelined
wavefront == hyperplane order, bit for bit), CUDA-graph replay == eager launches, run-to-run
determinism, and finite, bounded residuals over many steps.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def states(g):
    return [g.get_state(b) for b in range(g.nblk)]


def with_env(var, value, fn):
    old = os.environ.get(var)
    if value is None:
        os.environ.pop(var, None)
    else:
        os.environ[var] = value
    try:
        return fn()
    finally:
        if old is None:
            os.environ.pop(var, None)
        else:
            os.environ[var] = old


def test_config1_full_parity(gpu, oracle):
    """FP64 Euler channel bump, 129x65x17 nodes (131,072 cells), 8 LU-SGS steps."""
    from ocfd_b200 import cases
    p, case = cases.config1()
    o, g = oracle.OracleCase(p, case), gpu.Solver(p, case)
    for it in range(8):
        o.advance(1)
        g.advance(1)
        np.testing.assert_allclose(g.residual()[1][:5], o.residual()[1][:5], rtol=1e-11, err_msg="step %d" % it)
    A, B = o.get_state(0), g.get_state(0)
    assert (np.abs(A - B).max(axis=(0, 1, 2)) / np.abs(A).max(axis=(0, 1, 2))).max() <= 1e-11
    np.testing.assert_allclose(g.forces()[0], o.forces()[0], rtol=1e-10, atol=1e-14)
    g.close()
    o.close()


def test_config2_full_one_step_parity(gpu, oracle):
    """FP64 RANS-SA swept wing, 8 blocks, 2,088,960 cells: one LU-SGS step against the oracle
    (wall distance, metrics, residual, both sweeps, limiter, BC, halo, norms, forces)."""
    from ocfd_b200 import cases
    p, case = cases.config2()
    o, g = oracle.OracleCase(p, case), gpu.Solver(p, case)
    for b in range(o.nblk):
        a, _, _ = o.get_array(b, "dw")
        c, _, _ = g.get_array(b, "dw")
        assert np.abs(a - c).max() <= 1e-13 * np.abs(a).max()
    o.advance(1)
    g.advance(1)
    mo, ro = o.residual()
    mg, rg = g.residual()
    np.testing.assert_allclose(rg[:6], ro[:6], rtol=1e-11)
    np.testing.assert_allclose(mg[:6], mo[:6], rtol=1e-10)
    fo, fg = o.forces(), g.forces()
    np.testing.assert_allclose(fg[1:], fo[1:], rtol=1e-10, atol=1e-14)
    for b in range(o.nblk):
        A, B = o.get_state(b), g.get_state(b)
        assert (np.abs(A - B).max(axis=(0, 1, 2)) / np.abs(A).max(axis=(0, 1, 2))).max() <= 1e-11
    g.close()
    o.close()


def test_config2_wavefront_equals_hyperplanes(gpu):
    """The pipelined-wavefront LU-SGS gives bit for bit the hyperplane-order result."""
    from ocfd_b200 import cases
    p, case = cases.config2()
    a = gpu.Solver(p, case)
    b = with_env("OCFD_LUSGS_PLANES", "1", lambda: gpu.Solver(p, case))
    a.advance(3)
    b.advance(3)
    for x, y in zip(states(a), states(b)):
        assert np.array_equal(x, y)
    for blk in range(a.nblk):
        assert np.array_equal(a.get_array(blk, "DU")[0], b.get_array(blk, "DU")[0])
    a.close()
    b.close()


def test_config2_graph_equals_eager_and_deterministic(gpu):
    from ocfd_b200 import cases
    p, case = cases.config2()
    a = gpu.Solver(p, case)
    b = with_env("OCFD_NO_GRAPH", "1", lambda: gpu.Solver(p, case))
    c = gpu.Solver(p, case)
    for s in (a, b, c):
        s.advance(4)
    ra = a.residual()
    assert np.array_equal(ra[1], b.residual()[1]) and np.array_equal(ra[1], c.residual()[1])
    for x, y, z in zip(states(a), states(b), states(c)):
        assert np.array_equal(x, y) and np.array_equal(x, z)
    for s in (a, b, c):
        s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_config2_many_steps_stay_finite(gpu, precision):
    """200 steps of the benchmark loop from the impulsive start: finite, bounded residuals, no
    limiter event, finite forces."""
    from ocfd_b200 import cases
    p, case = cases.config2(precision=precision)
    g = gpu.Solver(p, case)
    g.advance(1)
    r0 = g.residual()[1][0]
    g.advance(199)
    r1 = g.residual()[1]
    assert np.all(np.isfinite(r1))
    assert r1[0] < 100.0 * r0
    for b in range(g.nblk):
        assert g.limiter_status(b) == (0, 0)
    _, cl, cd, _ = g.forces()
    assert np.isfinite(cl) and np.isfinite(cd)
    g.close()


def test_mixed_vs_fp64_forces_config2(gpu):
    """Mixed precision against FP64 on the full wing after 50 steps: CL, CD within 1e-3."""
    from ocfd_b200 import cases
    out = []
    for prec in (0, 1):
        p, case = cases.config2(precision=prec)
        g = gpu.Solver(p, case)
        g.advance(50)
        out.append(g.forces())
        g.close()
    (_, cl0, cd0, _), (_, cl1, cd1, _) = out
    assert abs(cl1 - cl0) <= 1e-3 * abs(cl0)
    assert abs(cd1 - cd0) <= 1e-3 * abs(cd0)


def test_config3_full_mixed_vs_fp64(gpu):
    """Config 3 stand-in: SST swept wing, 24 uneven blocks, 7,798,784 cells.  Mixed precision
    against FP64 after 20 LU-SGS steps: finite, CL / CD within 0.5 count (5e-5); the RK3 variant
    (CFL 0.5) advances 3 steps without NaN."""
    from ocfd_b200 import cases
    out = []
    for prec in (0, 1):
        p, case = cases.config3(precision=prec)
        assert len(case.dims) == 24 and case.ncells == 7798784
        g = gpu.Solver(p, case)
        g.advance(20)
        _, rms = g.residual()
        assert np.all(np.isfinite(rms))
        out.append(g.forces())
        g.close()
    (_, cl0, cd0, _), (_, cl1, cd1, _) = out
    assert abs(cl1 - cl0) <= 5e-5 and abs(cd1 - cd0) <= 5e-5, (cl0, cl1, cd0, cd1)
    p, case = cases.config3(time_method=3, cfl=0.5)
    g = gpu.Solver(p, case)
    g.advance(3)
    assert np.all(np.isfinite(g.residual()[1]))
    g.close()
