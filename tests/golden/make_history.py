"""Generates the long-horizon history fixtures in this folder from the CPU oracle (oracle/).

    python tests/golden/make_history.py [name ...]

Each fixture holds, for every iteration of a run, the residual norms (res_max, res_rms: the
values comput_max_Res_onemesh prints to Residual.dat, sub_time_advance.f90:330-403) and the force
coefficients (CL, CD, CS of comput_force, sub_Post.f90:4-265, as force.log records them), plus the
interior state checksums at the end.  The GPU tests replay the same run through the C-ABI and
compare the whole history, so a drift that grows slowly over thousands of iterations is caught,
not only the first steps.  The oracle's results are the same bits for any thread count, so the
fixtures do not depend on the machine that made them.

Runs:
  config1      the channel bump at full size (129x65x17, 131,072 cells), MUSCL3 + Roe, LU-SGS
               CFL 5, inviscid, 2000 iterations: the whole run of the configuration
  foil_sa      SA airfoil 65x17 (WENO5 + Roe, LU-SGS), 600 iterations
  wing8_sa     the reduced swept wing (8 blocks, SA, WENO5 + Roe), 200 iterations
  foil_sst_rk3 SST airfoil 65x17 (MUSCL3 + HLLC), three-stage RK3 at CFL 1.0, 300 steps
  bump_dual    the channel bump at a quarter size, dual time (dt 0.2, 3 inner LU-SGS iterations
               per physical step), 60 physical steps
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "opencfd-ec_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle_py as O  # noqa: E402
from golden.make_golden import interior_checksums  # noqa: E402
from ocfd_b200 import cases  # noqa: E402


def runs():
    return {
        "config1": (lambda: cases.config1(), 2000),
        "foil_sa": (lambda: cases.airfoil(ni=65, nj=17, scheme=7, flux=4, turb=2), 600),
        "wing8_sa": (lambda: cases.config2_small(), 200),
        "foil_sst_rk3": (lambda: cases.airfoil(ni=65, nj=17, scheme=5, flux=3, turb=3, time_method=3, cfl=1.0,
                                               kt_inf=1e-8, wt_inf=1e-5), 300),
        "bump_dual": (lambda: cases.config1(scale=0.25, time_method=-1, dt_global=0.2, step_inner_limit=3,
                                            res_inner_limit=1e-14), 60),
    }


def history(solver, steps):
    """Per-iteration norms and force coefficients of a solver object (oracle or GPU binding)."""
    rmax, rrms, coef = [], [], []
    for _ in range(steps):
        solver.advance(1)
        a, b = solver.residual()
        _, cl, cd, cs = solver.forces()
        rmax.append(a)
        rrms.append(b)
        coef.append((cl, cd, cs))
    return np.array(rmax), np.array(rrms), np.array(coef)


def make(name):
    make_case, steps = runs()[name]
    p, case = make_case()
    o = O.OracleCase(p, case)
    t0 = time.time()
    rmax, rrms, coef = history(o, steps)
    chk = np.stack([interior_checksums(o.get_state(b), case.dims[b]) for b in range(o.nblk)])
    o.close()
    np.savez(os.path.join(HERE, "history_%s.npz" % name), res_max=rmax, res_rms=rrms, clcdcs=coef, state_checksums=chk,
             steps=np.array(steps))
    print("wrote history_%s.npz: %d iterations in %.0f s, rms(rho) %.3e -> %.3e" % (name, steps, time.time() - t0, rrms[0, 0], rrms[-1, 0]))


def main(names):
    O.build()
    for n in names or list(runs()):
        make(n)


if __name__ == "__main__":
    main(sys.argv[1:])
