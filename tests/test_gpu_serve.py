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


def test_failing_request_leaves_the_others_untouched(gpu):
    """A request whose restart state holds a NaN fails on its first read-back (OCFD_ERR_NAN); it
    ends as an "error" result with the message, its handle is closed and its memory released,
    and every other request of the mix gives the same result as alone (bit for bit)."""
    import copy

    import torch
    from ocfd_b200 import capi
    from ocfd_b200.serve import Request, Server
    base = reqs()
    p, c = base[1].params, base[1].case
    s = capi.Solver(p, c)
    s.advance(3)
    state = [s.get_state(b) for b in range(s.nblk)]
    s.close()
    state[0][3 + 1, 3 + 5, 3 + 7, 0] = float("nan")
    bad = Request(9, p, c, 0.02, 300, state)
    free0 = torch.cuda.mem_get_info()[0]
    mix = Server(chunk=50).run(copy.copy(base) + [bad])
    assert len(mix) == 5
    r_bad = [r for r in mix if r.rid == 9][0]
    assert r_bad.converged == "error" and "NaN" in r_bad.error, r_bad.error
    for r in mix:
        if r.rid == 9:
            continue
        alone = Server(chunk=50).run([x for x in reqs() if x.rid == r.rid])[0]
        assert r.converged != "error"
        assert np.array_equal(alone.rms, r.rms) and alone.cl == r.cl and alone.cd == r.cd
    # every handle of the run was closed: the device memory is back
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)


def sweep_reqs(max_iters=300):
    """Four Mach / AoA points on one airfoil mesh and one request on another mesh."""
    from ocfd_b200 import cases
    from ocfd_b200.serve import Request
    its = [cases.airfoil(ni=65, nj=17, ma=ma, aoa=aoa, precision=1) for ma, aoa in ((0.5, 1.0), (0.6, 2.0), (0.7, 0.0), (0.55, 3.0))]
    its.append(cases.airfoil(ni=81, nj=21, m=0.03, ma=0.6, aoa=1.5, precision=1))
    arr = [0.0, 0.0, 0.05, 0.3, 0.1]
    return [Request(q, p, c, arr[q], max_iters) for q, (p, c) in enumerate(its)]


def test_slot_server_same_alone_and_in_the_mix(gpu):
    """Continuous batching inside batched steps (SlotServer): with two slots per mesh, the third
    and fourth requests on the first mesh wait for a slot and enter a running batch through
    ocfd_reset_solve; every result equals the same request run alone, bit for bit."""
    from ocfd_b200.serve import SlotServer
    mix = SlotServer(slots=2, chunk=50).run(sweep_reqs())
    assert len(mix) == 5 and all(r.converged != "error" for r in mix)
    for r in mix:
        alone = SlotServer(slots=2, chunk=50).run([x for x in sweep_reqs() if x.rid == r.rid])[0]
        assert alone.iters == r.iters and alone.converged == r.converged
        assert np.array_equal(alone.rms, r.rms)
        assert alone.cl == r.cl and alone.cd == r.cd
