"""The oracle's results do not depend on its host thread count.

The CPU baseline is timed on all host threads and on one (`cpu_baseline.single_thread` in the
bench line); both must compute the same thing.  The oracle's thread pool splits each loop into
contiguous chunks, one per thread, and every reduction (norms, forces) runs in a fixed order, so
the state, the norms and the forces are the same bits for any thread count.
"""
import numpy as np


def test_oracle_bits_independent_of_thread_count(oracle):
    import oracle_py
    from ocfd_b200 import cases
    n0 = oracle_py.threads()
    out = {}
    try:
        for nt in (1, 3, 8):
            assert oracle_py.set_threads(nt) == nt
            p, case = cases.config2_small()
            o = oracle.OracleCase(p, case)
            o.advance(3)
            U = [o.get_state(b).copy() for b in range(o.nblk)]
            rmax, rrms = o.residual()
            ft, cl, cd, cs = o.forces()
            o.close()
            out[nt] = (U, rmax, rrms, ft, cl, cd)
    finally:
        oracle_py.set_threads(n0)
    U1, m1, r1, f1, cl1, cd1 = out[1]
    for nt in (3, 8):
        U, m, r, f, cl, cd = out[nt]
        assert all(np.array_equal(a.view(np.uint64), b.view(np.uint64)) for a, b in zip(U, U1))
        assert np.array_equal(m, m1) and np.array_equal(r, r1)
        assert np.array_equal(np.asarray(f), np.asarray(f1)) and cl == cl1 and cd == cd1
