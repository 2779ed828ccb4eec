"""Block-sharded solves on the GPU (ocfd_create_part): n ranks as host threads of one process on
one GPU (ThreadComm: the exchange buffers move by device copies, the waits are host barriers with
a timeout, no kernel waits on another rank).  Each rank's blocks must equal the same blocks of the
unsharded solve bit for bit after every step (LU-SGS in FP64 and mixed precision, RK3, dual time),
and the all-reduced norms and forces must equal the unsharded ones up to the summation order
(1e-12)."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_sharded(p, case, owner, nrank, steps):
    from ocfd_b200.shard import ShardedSolver, ThreadComm
    hub = ThreadComm(nrank, timeout=300)
    out, err = [None] * nrank, [None] * nrank

    def run(r):
        try:
            import torch
            torch.cuda.set_device(0)
            s = ShardedSolver(p, case, owner, r, hub.comm(r))
            hist = []
            for _ in range(steps):
                k, _ = s.advance(1)
                hist.append((k, s.residual(), s.forces()))
            out[r] = (s.blocks, [s.get_state(b) for b in range(s.nblk)], hist, s.launches_per_step())
            s.close()
        except BaseException as e:  # noqa: BLE001 - reported below
            err[r] = e
            hub.bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(nrank)]
    for t in th:
        t.start()
    for t in th:
        t.join(600)
    for e in err:
        if e is not None:
            raise e
    return out


def _cases():
    from ocfd_b200 import cases
    return {
        "wing8_sa_lusgs": (lambda: cases.config2_small(), 2),
        "wing8_sa_lusgs_3ranks": (lambda: cases.config2_small(), 3),
        "wing8_sa_lusgs_mixed": (lambda: cases.config2_small(precision=1), 2),
        "bump2_rk3": (lambda: cases.config1(scale=0.25, cuts_i=(12,), time_method=3, cfl=1.0), 2),
        "bump2_dual": (lambda: cases.config1(scale=0.25, cuts_i=(12,), time_method=-1, dt_global=0.2, step_inner_limit=3,
                                             res_inner_limit=1e-14), 2),
    }


@pytest.mark.parametrize("name", list(_cases()))
def test_sharded_equals_unsharded(gpu, name):
    from ocfd_b200.shard import partition
    make, nrank = _cases()[name]
    p, case = make()
    owner = partition(case.dims, nrank)
    assert len(set(owner)) == nrank
    steps = 4
    g = gpu.Solver(p, case)
    ref = []
    for _ in range(steps):
        k, _ = g.advance(1)
        ref.append((k, g.residual(), g.forces()))
    ref_state = [g.get_state(b) for b in range(g.nblk)]
    g.close()
    out = _run_sharded(p, case, owner, nrank, steps)
    seen = []
    for r in range(nrank):
        blocks, states, hist, _ = out[r]
        assert all(owner[b] == r for b in blocks)
        seen += blocks
        for lb, gb in enumerate(blocks):
            assert np.array_equal(states[lb], ref_state[gb]), "rank %d block %d" % (r, gb)
        for (k, (mx, rms), (ft, cl, cd, cs)), (k0, (mx0, rms0), (ft0, cl0, cd0, cs0)) in zip(hist, ref):
            assert k == k0
            assert np.array_equal(mx, mx0)
            np.testing.assert_allclose(rms, rms0, rtol=1e-12, atol=0)
            np.testing.assert_allclose([cl, cd, cs], [cl0, cd0, cs0], rtol=1e-12, atol=1e-15)
    assert sorted(seen) == list(range(len(case.dims)))
