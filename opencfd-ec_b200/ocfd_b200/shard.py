"""Block-sharded solves: one case split over ranks by whole blocks, as the reference's MPI mode.

* ``partition(dims, nproc)`` -- the reference's automatic partition (sub_partation_mpi.f90:126-158):
  blocks ordered by node count, largest first (a selection sort that keeps the earlier of equal
  sizes in front), each given to the rank with the fewest nodes so far (the lowest such rank).
* ``plan(case, owner, rank)`` -- the exchange plan of one rank (``ocfd_part_plan``, host only).
* ``ShardedSolver`` -- this rank's blocks on the current GPU (``ocfd_create_part``); ``comm``
  carries the halo exchange and the all-reduce of norms and forces.
* ``TorchComm`` -- the comm over ``torch.distributed``: NCCL send/recv queued on the handle's
  stream for CUDA buffers (``batch_isend_irecv``), all-reduce of the host doubles.
* ``ThreadComm`` -- n ranks as host threads of one process sharing one GPU: buffers move by
  device copies between the ranks' handles; every wait is a host barrier with a timeout, no
  kernel waits on another rank.

The calls ``ocfd_create_part``, ``advance``, ``init_flow``, ``residual``, ``forces`` and ``profile``
are collective: every rank makes them in the same order.
"""
import ctypes
import threading

import numpy as np

from .capi import OcfdError, Solver, _dp, _ip, lib
from .params import OcfdParams

EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong))
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int)
OP_SUM, OP_MAX = 0, 1


class OcfdComm(ctypes.Structure):
    _fields_ = [("exchange", EXCHANGE_FN), ("allreduce", ALLREDUCE_FN), ("user", ctypes.c_void_p)]


def _bind():
    L = lib()
    if not getattr(L, "_part_bound", False):
        ip, lp = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)
        dpp = ctypes.POINTER(ctypes.POINTER(ctypes.c_double))
        L.ocfd_create_part.argtypes = [ctypes.POINTER(OcfdParams), ctypes.c_int, ip, dpp, ip, ip, dpp, ip, ctypes.c_int,
                                       ctypes.POINTER(OcfdComm), ctypes.POINTER(ctypes.c_void_p)]
        L.ocfd_part_blocks.argtypes = [ctypes.c_void_p, ip]
        L.ocfd_part_plan.argtypes = [ctypes.c_int, ip, ip, ip, ip, ctypes.c_int, ip, lp, lp]
        L._part_bound = True
    return L


def partition(dims, nproc):
    """owner[b] for every block: sub_partation_mpi.f90:126-158 (weights = node counts)."""
    g = [[nx * ny * nz, b] for b, (nx, ny, nz) in enumerate(dims)]
    for m in range(len(g)):                       # selection sort, largest first (lines 131-148)
        mg, g0 = m, g[m][0]
        for n in range(m + 1, len(g)):
            if g[n][0] > g0:
                g0, mg = g[n][0], n
        g[m], g[mg] = g[mg], g[m]
    load = [0] * nproc
    owner = [0] * len(dims)
    for w, b in g:                                # lightest rank so far (lines 150-162)
        m0 = 0
        for mp in range(nproc):
            if load[mp] < load[m0]:
                m0 = mp
        load[m0] += w
        owner[b] = m0
    return owner


def _flat(case):
    nijk, xyz, nsub, inc = case.flat()
    return (np.ascontiguousarray(nijk, dtype=np.int32), [np.ascontiguousarray(a, dtype=np.float64) for a in xyz],
            np.ascontiguousarray(nsub, dtype=np.int32), np.ascontiguousarray(inc, dtype=np.int32))


def plan(case, owner, rank):
    """(peers, send_off, recv_off) of one rank, offsets in cells (host only)."""
    L = _bind()
    nijk, _, nsub, inc = _flat(case)
    own = np.ascontiguousarray(owner, dtype=np.int32)
    n = L.ocfd_part_plan(len(case.dims), _ip(nijk), _ip(nsub), _ip(inc), _ip(own), rank, None, None, None)
    if n < 0:
        raise OcfdError(n, "ocfd_part_plan failed")
    peers = np.zeros(max(n, 1), dtype=np.int32)
    so, ro = np.zeros(n + 1, dtype=np.int64), np.zeros(n + 1, dtype=np.int64)
    L.ocfd_part_plan(len(case.dims), _ip(nijk), _ip(nsub), _ip(inc), _ip(own), rank, _ip(peers),
                     so.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), ro.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
    return peers[:n].tolist(), so.tolist(), ro.tolist()


class _CudaBuf:
    """A device range seen through __cuda_array_interface__ (zero copy into torch)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False), "version": 2}


def device_view(ptr, n):
    import torch
    if n == 0:
        return torch.empty(0, dtype=torch.float64, device="cuda")
    return torch.as_tensor(_CudaBuf(ptr, n), device="cuda")


def exchange_segments(send, send_off, recv, recv_off, peers, group=None):
    """send[send_off[q]:send_off[q+1]] -> rank peers[q], recv[recv_off[q]:recv_off[q+1]] <- it;
    one batch of point-to-point operations (NCCL or gloo), waited for on the current stream."""
    import torch.distributed as dist
    ops = []
    for q, peer in enumerate(peers):
        a, b, c, d = send_off[q], send_off[q + 1], recv_off[q], recv_off[q + 1]
        if b > a:
            ops.append(dist.P2POp(dist.isend, send[a:b], peer, group))
        if d > c:
            ops.append(dist.P2POp(dist.irecv, recv[c:d], peer, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class _CommBase:
    """Holds the ctypes callbacks (they must outlive the handle) and turns exceptions into -1."""

    def __init__(self):
        self.error = None
        self._ex = EXCHANGE_FN(self._exchange_cb)
        self._ar = ALLREDUCE_FN(self._allreduce_cb)
        self.struct = OcfdComm(self._ex, self._ar, None)

    def _exchange_cb(self, user, stream, npeer, peers, send, send_off, recv, recv_off):
        try:
            pe = [peers[q] for q in range(npeer)]
            so = [send_off[q] for q in range(npeer + 1)]
            ro = [recv_off[q] for q in range(npeer + 1)]
            self.exchange(stream, pe, ctypes.cast(send, ctypes.c_void_p).value or 0, so,
                          ctypes.cast(recv, ctypes.c_void_p).value or 0, ro)
            return 0
        except Exception as e:  # reported through OCFD_ERR_COMM
            self.error = e
            return -1

    def _allreduce_cb(self, user, buf, n, op):
        try:
            a = np.ctypeslib.as_array(buf, shape=(n,))
            a[:] = self.allreduce(a.copy(), op)
            return 0
        except Exception as e:
            self.error = e
            return -1


class TorchComm(_CommBase):
    """Exchange and all-reduce over the default torch.distributed group (NCCL: device buffers
    directly; the all-reduce moves the few host doubles through a device tensor)."""

    def __init__(self, group=None):
        super().__init__()
        self.group = group

    def exchange(self, stream, peers, send_ptr, send_off, recv_ptr, recv_off):
        import torch
        s = torch.cuda.ExternalStream(stream)
        with torch.cuda.stream(s):
            exchange_segments(device_view(send_ptr, send_off[-1]), send_off, device_view(recv_ptr, recv_off[-1]), recv_off,
                              peers, self.group)

    def allreduce(self, a, op):
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.from_numpy(a).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == OP_SUM else dist.ReduceOp.MAX, group=self.group)
        return t.cpu().numpy()


class ThreadComm:
    """n ranks as threads of one process on one GPU.  comm(r) gives rank r's comm."""

    def __init__(self, n, timeout=120.0):
        self.n = n
        self.bar = threading.Barrier(n, timeout=timeout)
        self.slot = [None] * n

    def comm(self, rank):
        return _ThreadRankComm(self, rank)


class _ThreadRankComm(_CommBase):
    def __init__(self, hub, rank):
        super().__init__()
        self.hub, self.rank = hub, rank

    def exchange(self, stream, peers, send_ptr, send_off, recv_ptr, recv_off):
        import torch
        torch.cuda.ExternalStream(stream).synchronize()          # this rank's pack is complete
        self.hub.slot[self.rank] = (peers, send_ptr, send_off)
        self.hub.bar.wait()
        recv = device_view(recv_ptr, recv_off[-1])
        for q, peer in enumerate(peers):
            pp, sp, so = self.hub.slot[peer]
            k = pp.index(self.rank)
            src = device_view(sp, so[-1])[so[k]:so[k + 1]]
            recv[recv_off[q]:recv_off[q + 1]].copy_(src)
        torch.cuda.synchronize()
        self.hub.bar.wait()                                       # no rank repacks before all copied

    def allreduce(self, a, op):
        self.hub.slot[self.rank] = a
        self.hub.bar.wait()
        parts = np.stack([self.hub.slot[r] for r in range(self.hub.n)])
        out = parts.sum(axis=0) if op == OP_SUM else parts.max(axis=0)
        self.hub.bar.wait()
        return out


class ShardedSolver(Solver):
    """This rank's blocks of a case; block numbers in get_state / set_state / get_array are local
    (``blocks`` maps them to the case's numbering)."""

    def __init__(self, params, case, owner, rank, comm, dw=None):
        L = _bind()
        self.cases = [case]
        self.case = case
        self.params = params.copy()
        self.params_list = [self.params]
        nijk, xyz, nsub, inc = _flat(case)
        own = np.ascontiguousarray(owner, dtype=np.int32)
        self._keep = (nijk, xyz, nsub, inc, own)
        self.comm = comm
        xyz_ptrs = (ctypes.POINTER(ctypes.c_double) * len(xyz))(*[_dp(a) for a in xyz])
        dwp = None
        if dw is not None:
            self._dw = [np.ascontiguousarray(d, dtype=np.float64) for d in dw]
            dwp = (ctypes.POINTER(ctypes.c_double) * len(dw))(*[_dp(a) for a in self._dw])
        h = ctypes.c_void_p()
        rc = L.ocfd_create_part(ctypes.byref(self.params), len(xyz), _ip(nijk), xyz_ptrs, _ip(nsub), _ip(inc), dwp, _ip(own),
                                rank, ctypes.byref(comm.struct), ctypes.byref(h))
        if rc != 0:
            raise OcfdError(rc, "ocfd_create_part failed" + ("" if comm.error is None else ": %r" % (comm.error,)))
        self.h = h
        n = L.ocfd_part_blocks(h, None)
        ids = np.zeros(n, dtype=np.int32)
        L.ocfd_part_blocks(h, _ip(ids))
        self.blocks = ids.tolist()
        self.nblk = n
        self.nsolve = 1
        self.blk0 = np.array([0, n])
        self.dims = [case.dims[g] for g in self.blocks]
        self.nvar = int(self.params.nvar)
        self.rank = rank
