"""Generates the golden fixtures in this folder from the CPU oracle (oracle/).

    python tests/golden/make_golden.py

The oracle restates the reference algorithm line by line; the reference ships no test vectors
and cannot be built here (Fortran, no compiler), so these fixtures pin the oracle against itself
(regression) and give the GPU tests committed vectors to compare against.  Inputs are seeded.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "opencfd-ec_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle_py as O  # noqa: E402
from cases_small import GOLDEN_CASES, GOLDEN_STEPS, small_cases  # noqa: E402

FLUXES = (1, 2, 3, 4, 5, 6)
SCHEMES = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 20)


def interior_checksums(U, dims):
    nx, ny, nz = dims
    I = U[4:nz + 3, 4:ny + 3, 4:nx + 3, :]
    return np.stack([I.sum(axis=(0, 1, 2)), (I * I).sum(axis=(0, 1, 2))])


def run_case(name, steps=GOLDEN_STEPS):
    p, case = small_cases()[name]()
    o = O.OracleCase(p, case)
    rmax, rrms = [], []
    for _ in range(steps):
        o.advance(1)
        a, b = o.residual()
        rmax.append(a)
        rrms.append(b)
    ft, cl, cd, cs = o.forces()
    chk = np.stack([interior_checksums(o.get_state(b), case.dims[b]) for b in range(o.nblk)])
    o.close()
    return dict(res_max=np.array(rmax), res_rms=np.array(rrms), ft=ft, clcdcs=np.array([cl, cd, cs]), state_checksums=chk)


def flux_vectors(seed=11, n=48):
    rng = np.random.default_rng(seed)
    QL = np.stack([rng.uniform(0.3, 2.0, n), rng.uniform(-1.5, 1.5, n), rng.uniform(-0.5, 0.5, n),
                   rng.uniform(-0.5, 0.5, n), rng.uniform(0.2, 2.0, n)], axis=1)
    QR = QL * rng.uniform(0.8, 1.25, (n, 5))
    F = np.array([[O.flux_1d(QL[q], QR[q], 1.4, f) for q in range(n)] for f in FLUXES])
    return dict(QL=QL, QR=QR, fluxes=np.array(FLUXES), F=F)


def scheme_vectors(seed=12, n=32):
    rng = np.random.default_rng(seed)
    U8 = rng.uniform(-1.0, 1.0, (n, 8)).cumsum(axis=1)
    LR = np.array([[O.scheme(U8[q], s) for q in range(n)] for s in SCHEMES])
    return dict(U8=U8, schemes=np.array(SCHEMES), LR=LR)


def main():
    O.build()
    np.savez(os.path.join(HERE, "flux_1d.npz"), **flux_vectors())
    np.savez(os.path.join(HERE, "schemes.npz"), **scheme_vectors())
    for name in GOLDEN_CASES:
        np.savez(os.path.join(HERE, "case_%s.npz" % name), **run_case(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
