"""Config 3 as the configuration states it, on the CPU restatement of the reference (oracle/).

The configuration asks for the swept wing with an ellipsoidal fuselage, RANS-SST, MUSCL3 with the
HLLC flux, LU-SGS, and an RK3 variant at CFL 1.5.  On the reduced wing-body (24 blocks, the same
generator as the full case) the reference algorithm diverges in both forms:
  * HLLC + LU-SGS: a NaN within the first ten iterations.  The reference's HLLC carries the right
    state's v into the right star state's w-momentum (sub_flux_split.f90:67), which on a 3-D wing
    injects spanwise momentum at every face whose tangential velocities differ;
  * RK3 at CFL 1.5 (HLLC or Roe): a NaN at the first step, in the far field beyond the tip, with
    the SST model only (Euler, laminar and SA run at the same CFL).
The stand-in the benchmark times (Roe + LU-SGS at CFL 1, RK3 at CFL 0.5) runs on the same mesh.
"""
import numpy as np
import pytest

from ocfd_b200 import cases


def small(**over):
    return cases.config3_small(**over)


def run(oracle, p, case, steps):
    """Iterations until the first NaN (None if none within steps)."""
    o = oracle.OracleCase(p, case)
    try:
        for it in range(steps):
            o.advance(1)
            try:
                o.residual()
            except FloatingPointError:
                return it + 1
        return None
    finally:
        o.close()


def test_wingbody_mesh_has_the_fuselage():
    from ocfd_b200.meshgen import fuselage_lift
    p, case = small()
    # the root plane's wall section sits on the ellipsoid's side (z > 0), the far root plane at 0
    X = case.xyz[0]                          # blocks 0..3: the wall layer of the root span
    assert X[2, 0, 0].min() > 0.2            # wall nodes of the root section: lifted ~0.24-0.25
    Xf = case.xyz[8]                         # blocks 8..11: the outer layer, ending at the far field
    assert abs(Xf[2, 0, -1]).max() < 1e-12   # far field of the root plane: still on z = 0
    assert abs(fuselage_lift(np.array(0.5), np.array(0.0), **cases.FUSELAGE) - 0.25) < 1e-15


def test_as_specified_hllc_diverges(oracle):
    p, case = small(iflag_flux=3)
    n = run(oracle, p, case, 10)
    assert n is not None and n <= 10, n


def test_as_specified_rk3_cfl15_diverges(oracle):
    for flux in (3, 4):
        p, case = small(iflag_flux=flux, time_method=3, cfl=1.5)
        assert run(oracle, p, case, 3) == 1


def test_stand_in_runs(oracle):
    p, case = small()
    assert run(oracle, p, case, 20) is None
    p, case = small(time_method=3, cfl=0.5)
    assert run(oracle, p, case, 10) is None
