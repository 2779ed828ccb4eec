"""The oracle takes the branches the GPU branch-parity tests are meant to cover (CPU only).

The GPU tests in test_gpu_branches.py compare the CUDA path with the oracle on the cases of
branch_cases.py; these tests show, on the oracle alone, that each case really reaches its branch:
limited cells and the sticky IF_OverLimit flag (sub_limitflow.f90:152-171), the clamp of a cell
with no good neighbour (117-131), a negative reconstructed pressure with the positivity fallback
on (sub_Residual.f90:283-299) and a NaN with it off, and mu_t held at MUT_MAX * mu
(sub_Residual.f90:1387-1408).
"""
import numpy as np
import pytest

import branch_cases as BC


@pytest.mark.parametrize("name", list(BC.limiter_cases()))
def test_limiter_fires_and_sticks(oracle, name):
    p, case, warm, preps, steps = BC.limiter_cases()[name]()
    o = oracle.OracleCase(p, case)
    o.advance(warm)
    assert all(o.limiter_status(b) == (0, 0) for b in range(o.nblk)), "bounds crossed before the prepared state"
    BC.prepare(o, p, 0, preps)
    o.advance(1)
    for b in range(o.nblk):
        n, ov = o.limiter_status(b)
        if b in preps:
            # RK3 counts the limited cells of its last stage only; the first stage repaired them
            assert ov == 1 and (n > 0 or p.time_method == 3), (b, n, ov)
        else:
            assert (n, ov) == (0, 0), (b, n, ov)
    for _ in range(steps - 1):
        o.advance(1)
        for b in preps:
            assert o.limiter_status(b)[1] == 1     # IF_OverLimit stays set
    o.close()


def test_cell_without_good_neighbour_is_clamped(oracle):
    p, case, warm, preps, _ = BC.limiter_cases()["bump_euler"]()
    o = oracle.OracleCase(p, case)
    BC.prepare(o, p, warm, preps)
    o.advance(1)
    i, j, k = BC.CLUSTER_CENTRE
    assert o.get_state(0)[k + 3, j + 3, i + 3, 0] == p.ldmax    # d0 = Ldmax (sub_limitflow.f90:125)
    o.close()


@pytest.mark.parametrize("scheme", [2, 8, 7])
def test_positivity_fallback_is_reached(oracle, scheme):
    p, case, warm, preps, _ = BC.positivity_case(scheme)
    o = oracle.OracleCase(p, case)
    BC.prepare(o, p, warm, preps)
    U = o.get_state(0)
    d = U[..., 0]
    u, v, w = U[..., 1] / d, U[..., 2] / d, U[..., 3] / d
    pr = (U[..., 4] - 0.5 * d * (u * u + v * v + w * w)) * (p.gamma - 1.0)
    (i0, j, k), (i1, _, _) = BC.POCKET_CELLS
    f = i1          # the face between the two pocket cells; its stencil is cells f-4 .. f+3
    L, R = oracle.scheme(pr[k + 3, j + 3, f - 4 + 3:f + 4 + 3], scheme)
    assert L <= 1e-20 and R <= 1e-20, (L, R)
    o.advance(1)
    assert np.all(np.isfinite(o.residual()[1][:5]))
    q = p.copy()
    q.if_scheme_positivity = 0
    o2 = oracle.OracleCase(q, case)
    BC.prepare(o2, q, warm, preps)
    o2.advance(1)
    with pytest.raises(FloatingPointError):
        o2.residual()
    o.close()
    o2.close()


@pytest.mark.parametrize("turb", [2, 3])
def test_mut_max_binds(oracle, turb):
    p, case, warm, _, _ = BC.mut_max_case(turb)
    o = oracle.OracleCase(p, case)
    o.advance(warm)
    o.compute_residual(False)
    mu, _, _ = o.get_array(0, "mu")
    mt, _, _ = o.get_array(0, "mu_t")
    ratio = (mt[1:-1, 1:-1, 1:-1] / mu[1:-1, 1:-1, 1:-1]).max()
    assert abs(ratio - p.mut_max) <= 1e-12 * p.mut_max, ratio
    o.close()
