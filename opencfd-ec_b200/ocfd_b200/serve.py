"""Continuous-batching request loop over the C-ABI.

Requests (a case + its parameters) arrive over time.  The loop admits a waiting request as soon
as a slot is free and its device footprint (``ocfd_footprint``) fits in the HBM budget, keeps
every admitted solve resident on the device, and advances every admitted solve at its own pace:
``chunk`` iterations are queued on the handle's own stream (so the solves overlap on the GPU),
and as soon as that stream is idle the loop reads back the solve's residual norms and forces and
queues its next chunk, without waiting for larger solves in the mix.  A solve leaves as soon as it
converges (density-residual RMS down by ``drop`` from its first iteration, or |dCL| below
``dcl`` over the last ``dcl_window`` iterations) or reaches ``max_iters``; its memory is
released for the next admission.

A request whose solve fails (a NaN in its residual, a device wait that ran out, a CUDA error on
its handle) ends with ``converged == "error"`` and the message; its handle is closed and its
memory released, and the other solves go on.  If the loop itself is left by an exception, every
handle still open is closed.

The sequence of operations on one handle does not depend on the other solves in flight, so a
request's result is the same alone and in the mix (bit for bit).  No counterpart in the
reference, which runs one case per MPI job.
"""
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import capi


@dataclass
class Request:
    rid: int
    params: object
    case: object
    arrival: float = 0.0            # seconds after the loop starts
    max_iters: int = 5000
    state: Optional[list] = None    # initial state per block (Fortran layout, as a restart reads it)


@dataclass
class Result:
    rid: int
    cells: int
    arrival: float
    admitted: float
    finished: float
    iters: int
    converged: str                  # "residual", "cl", "max_iters", or "error"
    rms0: float
    rms: np.ndarray
    cl: float
    cd: float
    cl_hist: List[float] = field(default_factory=list)
    error: str = ""

    @property
    def latency(self):
        return self.finished - self.arrival


class _Active:
    def __init__(self, req, solver, admitted):
        import torch
        self.req, self.s, self.admitted = req, solver, admitted
        self.iters = 0
        self.rms0 = None
        self.cl_hist = []    # (iteration, CL) at every read-back
        self.stream = torch.cuda.ExternalStream(solver.stream())  # idle test without blocking


class Server:
    def __init__(self, hbm_budget: Optional[int] = None, max_active: int = 32, chunk: int = 50, drop: float = 1e-6,
                 dcl: float = 1e-4, dcl_window: int = 200, clock=time.perf_counter):
        self.hbm_budget = hbm_budget
        self.max_active = max_active
        self.chunk = chunk
        self.drop, self.dcl, self.dcl_window = drop, dcl, dcl_window
        self.clock = clock

    def _budget(self):
        if self.hbm_budget is not None:
            return self.hbm_budget
        import torch
        free, _ = torch.cuda.mem_get_info()
        return int(free * 0.9)

    def _start(self, r):
        """Handle, restart state and first iteration of request r."""
        s = capi.Solver(r.params, r.case)
        try:
            if r.state is not None:
                for b, U in enumerate(r.state):
                    s.set_state(b, U)
            s.advance(1)
        except Exception:
            s.close()
            raise
        return s

    def _done(self, a):
        _, rms = a.s.residual()
        _, cl, cd, _ = a.s.forces()
        a.cl_hist.append((a.iters, cl))
        if a.rms0 is None:
            a.rms0 = rms[0]
        if rms[0] <= self.drop * a.rms0:
            return "residual", rms, cl, cd
        old = [c for it, c in a.cl_hist if it <= a.iters - self.dcl_window]
        if old and a.iters >= self.dcl_window and abs(cl - old[-1]) < self.dcl and \
                all(abs(cl - c) < self.dcl for it, c in a.cl_hist if it >= a.iters - self.dcl_window):
            return "cl", rms, cl, cd
        if a.iters >= a.req.max_iters:
            return "max_iters", rms, cl, cd
        return None, rms, cl, cd

    def run(self, requests: List[Request]) -> List[Result]:
        pending = sorted(requests, key=lambda r: r.arrival)
        queue, active, results = [], [], []
        budget = self._budget()
        used = 0
        fp = {}
        t0 = self.clock()

        def failed(r, admitted, iters, err, a=None):
            nan = float("nan")
            results.append(Result(r.rid, r.case.ncells, r.arrival, admitted, self.clock() - t0, iters, "error",
                                  nan if a is None or a.rms0 is None else float(a.rms0), np.full(7, nan), nan, nan,
                                  [] if a is None else [c for _, c in a.cl_hist], str(err)))

        try:
            while pending or queue or active:
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.pop(0))
                # admission: FIFO, by free slot and device footprint
                while queue and len(active) < self.max_active:
                    r = queue[0]
                    need = fp.setdefault(r.rid, capi.footprint(r.params, r.case))
                    if used + need > budget:
                        if not active:
                            raise MemoryError("request %d needs %d bytes, budget %d" % (r.rid, need, budget))
                        break
                    queue.pop(0)
                    admitted = self.clock() - t0
                    try:
                        s = self._start(r)
                    except (capi.OcfdError, FloatingPointError) as e:
                        failed(r, admitted, 0, e)
                        continue
                    used += need
                    a = _Active(r, s, admitted)
                    a.iters = 1
                    active.append(a)
                if not active:
                    if pending:
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - (self.clock() - t0))))
                    continue
                # every solve whose queued chunk has finished is read back and given its next chunk;
                # the others keep running
                still, progressed = [], False
                for a in active:
                    if not a.stream.query():
                        still.append(a)
                        continue
                    progressed = True
                    try:
                        why, rms, cl, cd = self._done(a)
                        if why is None:
                            n = min(self.chunk, a.req.max_iters - a.iters)
                            a.s.advance(n)
                            a.iters += n
                            still.append(a)
                            continue
                    except (capi.OcfdError, FloatingPointError) as e:
                        failed(a.req, a.admitted, a.iters, e, a)
                    else:
                        fin = self.clock() - t0
                        results.append(Result(a.req.rid, a.req.case.ncells, a.req.arrival, a.admitted, fin, a.iters, why,
                                              float(a.rms0), rms.copy(), cl, cd, [c for _, c in a.cl_hist]))
                    a.s.close()
                    used -= fp[a.req.rid]
                active = still
                if not progressed:
                    time.sleep(0.0002)
        finally:
            for a in active:
                a.s.close()
        return sorted(results, key=lambda r: r.rid)


def mesh_key(case):
    """Identity of a request's mesh (block sizes and node coordinates): requests with the same key
    can share the slots of one batch handle."""
    import hashlib
    h = hashlib.sha1()
    for d, x in zip(case.dims, case.xyz):
        h.update(np.asarray(d, dtype=np.int64).tobytes())
        h.update(np.ascontiguousarray(x).tobytes())
    return h.hexdigest()


class _Pool:
    """One batch handle whose solves are slots for requests on one mesh."""

    def __init__(self, req, slots, admitted):
        import torch
        self.b = capi.Batch([(req.params, req.case)] * slots)
        self.stream = torch.cuda.ExternalStream(self.b.stream())
        self.req = [None] * slots           # the request in each slot (None: free)
        self.iters = [0] * slots
        self.rms0 = [None] * slots
        self.cl_hist = [[] for _ in range(slots)]
        self.admitted = [0.0] * slots
        self.req[0] = req
        self.admitted[0] = admitted
        self.busy = False                   # a chunk is queued


class SlotServer:
    """Continuous batching inside batched steps: requests on the same mesh (Mach / AoA / Re
    sweeps on one geometry) are admitted into free slots of one batch handle, whose step graph
    advances all of them in the same launches; a new request takes a free slot through
    ocfd_reset_solve while the other slots keep iterating.  A mesh seen for the first time gets
    a handle of `slots` solves (admission by device footprint, as Server); idle slots are stepped
    along with the others.  Every request is checked at the same points (every `chunk` of its
    own iterations) with the same convergence tests as Server, so its result is the same alone
    and in the mix (bit for bit)."""

    def __init__(self, slots=8, chunk=50, hbm_budget: Optional[int] = None, drop: float = 1e-6, dcl: float = 1e-4,
                 dcl_window: int = 200, clock=time.perf_counter):
        self.slots, self.chunk, self.hbm_budget = slots, chunk, hbm_budget
        self.drop, self.dcl, self.dcl_window = drop, dcl, dcl_window
        self.clock = clock

    def _check(self, P, q, rms, cl):
        P.cl_hist[q].append((P.iters[q], cl))
        if P.rms0[q] is None:
            P.rms0[q] = rms[0]
        if rms[0] <= self.drop * P.rms0[q]:
            return "residual"
        it, hist = P.iters[q], P.cl_hist[q]
        old = [c for i, c in hist if i <= it - self.dcl_window]
        if old and it >= self.dcl_window and abs(cl - old[-1]) < self.dcl and \
                all(abs(cl - c) < self.dcl for i, c in hist if i >= it - self.dcl_window):
            return "cl"
        if it >= P.req[q].max_iters:
            return "max_iters"
        return None

    def run(self, requests: List[Request]) -> List[Result]:
        pending = sorted(requests, key=lambda r: r.arrival)
        queue, results, pools, keys = [], [], {}, {}
        budget = self.hbm_budget
        if budget is None:
            import torch
            budget = int(torch.cuda.mem_get_info()[0] * 0.9)
        used = 0
        t0 = self.clock()

        def finish(P, q, why, rms, cl, cd, err=""):
            r = P.req[q]
            results.append(Result(r.rid, r.case.ncells, r.arrival, P.admitted[q], self.clock() - t0, P.iters[q], why,
                                  float("nan") if P.rms0[q] is None else float(P.rms0[q]), rms, cl, cd,
                                  [c for _, c in P.cl_hist[q]], err))
            P.req[q] = None

        try:
            while pending or queue or any(any(r is not None for r in P.req) for P in pools.values()):
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    r = pending.pop(0)
                    keys[r.rid] = mesh_key(r.case)
                    queue.append(r)
                # a mesh seen for the first time: a new handle of `slots` solves, by footprint
                for r in list(queue):
                    k = keys[r.rid]
                    if k in pools:
                        continue
                    need = self.slots * capi.footprint(r.params, r.case)
                    if used + need > budget:
                        continue
                    pools[k] = _Pool(r, self.slots, self.clock() - t0)
                    used += need
                    queue.remove(r)
                progressed = False
                for k, P in pools.items():
                    if P.busy and not P.stream.query():
                        continue
                    if P.busy:   # a chunk has finished: read back and check every occupied slot
                        progressed = True
                        _, rms = P.b.residual_all()
                        _, cl, cd, _ = P.b.forces_all()
                        for q in range(self.slots):
                            if P.req[q] is None:
                                continue
                            if not np.isfinite(rms[q][0]):
                                finish(P, q, "error", rms[q].copy(), float("nan"), float("nan"), "NaN in the residual")
                                continue
                            why = self._check(P, q, rms[q], cl[q])
                            if why is not None:
                                finish(P, q, why, rms[q].copy(), float(cl[q]), float(cd[q]))
                        P.busy = False
                    # queued requests on this mesh take the free slots
                    for r in list(queue):
                        if keys[r.rid] != k or None not in P.req:
                            continue
                        q = P.req.index(None)
                        P.b.reset_solve(q, r.params)
                        P.req[q], P.iters[q], P.rms0[q], P.cl_hist[q] = r, 0, None, []
                        P.admitted[q] = self.clock() - t0
                        queue.remove(r)
                    if any(r is not None for r in P.req):
                        P.b.advance(self.chunk)
                        for q in range(self.slots):
                            if P.req[q] is not None:
                                P.iters[q] += self.chunk
                        P.busy = True
                        progressed = True
                if not progressed:
                    time.sleep(0.0002)
        finally:
            for P in pools.values():
                P.b.close()
        return sorted(results, key=lambda r: r.rid)


def poisson_requests(items, rate=2.0, seed=2024, max_iters=5000):
    """Requests for the given (params, case) items with exponential inter-arrival times."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for q, (p, case) in enumerate(items):
        t += float(rng.exponential(1.0 / rate))
        out.append(Request(q, p, case, t, max_iters))
    return out


def summarize(results, wall_s):
    lat = np.array([r.latency for r in results])
    cells = sum(r.cells * r.iters for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "cell_updates_per_s": cells / wall_s, "wall_s": wall_s,
            "converged": {k: sum(1 for r in results if r.converged == k) for k in ("residual", "cl", "max_iters", "error")}}
