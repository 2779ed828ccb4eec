"""Mixed precision against FP64 at convergence.

The mixed form keeps the conserved-state accumulation, the LU-SGS diagonal and division, the
residual norms and the force integration in FP64, and evaluates reconstruction, fluxes, sources,
metrics, Res, dt and the spectral radii in FP32.  Its answer must stay within 0.5 count (5e-5) of
the FP64 answer in CL and CD once both have converged, not only after a few iterations.

The solves are config-4 airfoils (the 64-airfoil batch, seed 1234: SA, AUSMPW + MUSCL3,
Re 6e6): those whose FP64 CL settles within 8000 iterations (it moves by less than 0.1 count over
the last 400), subsonic to M 0.74.  They run as one batch in each precision (a solve's result is
the same alone and in a batch).  Every one of them must have settled, and each must agree within
0.5 count in CL and in CD.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ITERS, WINDOW, CHUNK = 8000, 400, 200
COUNT = 1e-4
SETTLED = (7, 9, 29, 40, 44, 48, 59)   # indices in cases.config4_batch(n=64)


def items(precision):
    from ocfd_b200 import cases
    allq = cases.config4_batch(n=64, precision=precision)
    return [allq[q] for q in SETTLED]


def cl_cd_history(gpu, precision):
    b = gpu.Batch(items(precision))
    cl, cd = [], []
    for _ in range(ITERS // CHUNK):
        b.advance(CHUNK)
        _, c_l, c_d, _ = b.forces_all()
        cl.append(c_l.copy())
        cd.append(c_d.copy())
    b.close()
    return np.array(cl), np.array(cd)


def test_mixed_within_half_a_count_at_convergence(gpu):
    cl64, cd64 = cl_cd_history(gpu, 0)
    cl32, cd32 = cl_cd_history(gpu, 1)
    w = WINDOW // CHUNK
    moving = np.abs(cl64[-1] - cl64[-1 - w]) / COUNT
    assert np.all(moving < 0.1), moving                  # the FP64 answers have converged
    dcl = np.abs(cl32[-1] - cl64[-1]) / COUNT
    dcd = np.abs(cd32[-1] - cd64[-1]) / COUNT
    assert dcl.max() <= 0.5 and dcd.max() <= 0.5, (dcl, dcd)
