"""The continuous-batching request loop (ocfd_b200.serve): admission by slot and HBM footprint,
overlapping solves, and every result the same alone and in the mix (bit for bit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def reqs(max_iters=300):
    from ocfd_b200 import cases
    from ocfd_b200.serve import Request
    its = [cases.airfoil(ni=65, nj=17, ma=0.6, aoa=1.0, precision=1),
           cases.airfoil(ni=81, nj=21, ma=0.7, aoa=2.5, m=0.03, precision=1),
           cases.airfoil(ni=49, nj=17, ma=0.5, aoa=-1.0, t=0.10, precision=1),
           cases.airfoil(ni=97, nj=25, ma=0.75, aoa=0.5, precision=1)]
    arr = [0.0, 0.0, 0.05, 0.1]
    return [Request(q, p, c, arr[q], max_iters) for q, (p, c) in enumerate(its)]


def test_results_same_alone_and_in_the_mix(gpu):
    from ocfd_b200.serve import Server
    mix = Server(chunk=50).run(reqs())
    assert len(mix) == 4
    for r in mix:
        alone = Server(chunk=50).run([x for x in reqs() if x.rid == r.rid])[0]
        assert alone.iters == r.iters and alone.converged == r.converged
        assert np.array_equal(alone.rms, r.rms)
        assert alone.cl == r.cl and alone.cd == r.cd
        assert alone.cl_hist == r.cl_hist


def test_admission_by_footprint(gpu):
    """With an HBM budget for two of the four solves, at most two are resident at a time and all
    four finish; later arrivals wait and are admitted when memory frees up."""
    from ocfd_b200 import capi
    from ocfd_b200.serve import Server
    rs = reqs(max_iters=150)
    fps = sorted(capi.footprint(r.params, r.case) for r in rs)
    budget = fps[-1] + fps[-2]
    out = Server(hbm_budget=budget, chunk=50).run(rs)
    assert len(out) == 4
    events = sorted([(r.admitted, 1) for r in out] + [(r.finished, -1) for r in out], key=lambda e: (e[0], e[1]))
    live = peak = 0
    for _, d in events:
        live += d
        peak = max(peak, live)
    assert peak <= 2
    assert all(r.iters == 150 or r.converged != "max_iters" for r in out)
