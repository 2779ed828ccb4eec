"""The rarely taken, default-on branches on the CUDA path (through the C-ABI) against the oracle.

The cases (branch_cases.py) prepare a state on the host, write it with set_state on both sides,
and advance them together.  test_oracle_branches.py shows on the CPU that each case reaches its
branch; here every iteration must match: residual norms within 1e-11 relative (summation order
differs), the limited-cell count and IF_OverLimit of every block equal, forces within 1e-10, the
state within 1e-11 of its scale at the end.  The branches:
  limit_flow_U repair, clamp and sticky IF_OverLimit (sub_limitflow.f90:24-176), limit_flow_SA
  (182-231), UD1 / no viscous flux / dt x 0.1 under IF_OverLimit (sub_Residual.f90:227-245,
  734-750; sub_time_acceleraction.f90:74-79), the positivity fallback (sub_Residual.f90:283-299)
  and MUT_MAX (sub_Residual.f90:1387-1408).
"""
import numpy as np
import pytest

import branch_cases as BC
from test_gpu_parity import overlap, state_err

pytestmark = pytest.mark.gpu


def run_pair(gpu, oracle, p, case, warm, preps, steps):
    o, g = oracle.OracleCase(p, case), gpu.Solver(p, case)
    BC.prepare(o, p, warm, preps)
    BC.prepare(g, p, warm, preps)
    assert state_err(o, g) <= 1e-11
    statuses = []
    for it in range(steps):
        o.advance(1)
        g.advance(1)
        mo, ro = o.residual()
        mg, rg = g.residual()
        nv = p.nvar
        np.testing.assert_allclose(rg[:nv], ro[:nv], rtol=1e-11, atol=1e-300, err_msg="rms step %d" % it)
        np.testing.assert_allclose(mg[:nv], mo[:nv], rtol=1e-10, atol=1e-300, err_msg="max step %d" % it)
        so = [o.limiter_status(b) for b in range(o.nblk)]
        sg = [g.limiter_status(b) for b in range(g.nblk)]
        assert sg == so, "limiter status step %d: gpu %s oracle %s" % (it, sg, so)
        statuses.append(so)
    fo, fg = o.forces(), g.forces()
    np.testing.assert_allclose(fg[0], fo[0], rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(fg[1:], fo[1:], rtol=1e-10, atol=1e-14)
    assert state_err(o, g) <= 1e-11
    return o, g, statuses


@pytest.mark.parametrize("name", list(BC.limiter_cases()))
def test_limiter_branches_match_oracle(gpu, oracle, name):
    p, case, warm, preps, steps = BC.limiter_cases()[name]()
    o, g, statuses = run_pair(gpu, oracle, p, case, warm, preps, steps)
    for b in preps:      # the prepared blocks went through the repair and stayed in OverLimit mode
        assert statuses[0][b][1] == 1 and statuses[-1][b][1] == 1
    if name == "wing8_sa":
        assert any(statuses[-1][b][1] == 0 for b in range(o.nblk))
    g.close()
    o.close()


@pytest.mark.parametrize("scheme", [2, 8, 7])
def test_positivity_fallback_matches_oracle(gpu, oracle, scheme):
    p, case, warm, preps, steps = BC.positivity_case(scheme)
    o, g, _ = run_pair(gpu, oracle, p, case, warm, preps, steps)
    g.close()
    o.close()


@pytest.mark.parametrize("turb", [2, 3])
def test_mut_max_matches_oracle(gpu, oracle, turb):
    p, case, warm, preps, steps = BC.mut_max_case(turb)
    o, g, _ = run_pair(gpu, oracle, p, case, warm, preps, steps)
    o.compute_residual(False)
    g.compute_residual(False)
    for name in ("mu_t", "Res"):
        a, lo, _ = o.get_array(0, name)
        c, lo2, _ = g.get_array(0, name)
        a = overlap(a, lo, c, lo2)
        assert np.abs(a - c).max() <= 1e-11 * np.abs(a).max(), name
    g.close()
    o.close()
