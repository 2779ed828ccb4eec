"""Block sharding on CPU: the reference's automatic partition, the per-rank exchange plans of the
C-ABI (host-only ocfd_part_plan) checked for agreement between world_size-2 gloo ranks and against
the case's interface table, the point-to-point exchange and the all-reduce of the torch.distributed
comm over gloo, and the thread-rank comm's all-reduce."""
import os
import socket
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_partition_follows_reference_greedy():
    """sub_partation_mpi.f90:126-162 by hand: order b1, b3, b2, b0, b4 (300, 300, 200, 100, 50
    nodes; the earlier of equal sizes first), each to the lightest rank (the lower of equal ones)."""
    from ocfd_b200.shard import partition
    dims = [(10, 10, 1), (10, 10, 3), (10, 10, 2), (10, 10, 3), (5, 10, 1)]
    assert partition(dims, 2) == [1, 0, 0, 1, 1]
    assert partition(dims, 1) == [0] * 5
    owner = partition(dims, 5)
    assert sorted(owner) == [0, 1, 2, 3, 4]


def _inter_rank_cells(case, owner):
    """cells each ordered pair of ranks exchanges, from the case's .inc records (LAP ghost layers
    of the target side of every interface between blocks on different ranks)."""
    _, _, nsub, inc = case.flat()
    inc = np.asarray(inc).reshape(-1, 21)
    out = {}
    t = 0
    for b, n in enumerate(nsub):
        for _ in range(n):
            r = inc[t]
            t += 1
            if r[6] >= 0:
                continue
            nb = r[15] - 1
            if owner[b] == owner[nb]:
                continue
            lo = [r[9], r[11], r[13]]
            hi = [r[10] - 1, r[12] - 1, r[14] - 1]
            d = (r[16] - 1) % 3
            if r[16] <= 3:
                lo[d] -= 4
            hi[d] = lo[d] + 3
            cells = int(np.prod([hi[q] - lo[q] + 1 for q in range(3)]))
            key = (owner[b], owner[nb])
            out[key] = out.get(key, 0) + cells
    return out


def test_plan_matches_interface_table():
    from ocfd_b200 import cases
    from ocfd_b200.shard import partition, plan
    p, case = cases.config2_small()
    for nproc in (2, 3):
        owner = partition(case.dims, nproc)
        want = _inter_rank_cells(case, owner)
        for rank in range(nproc):
            peers, so, ro = plan(case, owner, rank)
            assert peers == sorted(peers) and rank not in peers
            for q, peer in enumerate(peers):
                assert so[q + 1] - so[q] == want.get((rank, peer), 0)
                assert ro[q + 1] - ro[q] == want.get((peer, rank), 0)
            assert so[-1] == sum(v for (a, _), v in want.items() if a == rank)


def test_plan_refuses_thin_blocks_across_ranks():
    """Blocks thinner than LAP cells across an interface between ranks would make the exchange
    order matter (their copies read ghost cells other copies write): refused."""
    from meshes import wavy_box
    from ocfd_b200.capi import OCFD_ERR_UNSUPPORTED, OcfdError
    from ocfd_b200.shard import plan
    case = wavy_box(nx=21, ny=11, nz=7, cuts=(4, 12))          # blocks of 3, 8 and 9 cells in i
    with pytest.raises(OcfdError) as e:
        plan(case, [0, 1, 1], 0)
    assert e.value.code == OCFD_ERR_UNSUPPORTED
    peers, so, ro = plan(case, [0, 0, 1], 0)                   # the thin block's interface stays on rank 0
    assert peers == [1] and so[1] == ro[1] == 10 * 6 * 4


def _rank_main(rank, world, port, out_dir):
    import sys
    for p in (os.path.join(ROOT, "opencfd-ec_b200"), os.path.join(ROOT, "oracle"), ROOT):
        sys.path.insert(0, p)
    import datetime

    import torch
    import torch.distributed as dist

    from ocfd_b200 import cases
    from ocfd_b200.shard import OP_MAX, OP_SUM, TorchComm, exchange_segments, partition, plan
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    _, case = cases.config2_small()
    owner = partition(case.dims, world)
    peers, so, ro = plan(case, owner, rank)
    # the two ranks' plans line up: what one sends to the other is what the other receives
    allp = [None] * world
    dist.all_gather_object(allp, (peers, so, ro))
    ok = True
    for q, peer in enumerate(peers):
        pp, pso, pro = allp[peer]
        k = pp.index(rank)
        ok &= (so[q + 1] - so[q]) == (pro[k + 1] - pro[k]) and (ro[q + 1] - ro[q]) == (pso[k + 1] - pso[k])
    # exchange of the buffers (NV = 6 doubles per cell), values tagged by sender and position
    nv = 6
    send = torch.arange(so[-1] * nv, dtype=torch.float64) + 1e6 * (rank + 1)
    recv = torch.full((ro[-1] * nv,), -1.0, dtype=torch.float64)
    exchange_segments(send, [v * nv for v in so], recv, [v * nv for v in ro], peers)
    comm = TorchComm()
    s = comm.allreduce(np.array([rank + 1.0, 2.0 * rank]), OP_SUM)
    m = comm.allreduce(np.array([rank + 1.0, -rank]), OP_MAX)
    np.savez(os.path.join(out_dir, "rank%d.npz" % rank), ok=ok, recv=recv.numpy(), ro=np.array(ro), s=s, m=m,
             peers=np.array(peers))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_exchange_over_gloo(tmp_path):
    world, port = 2, _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    r = [np.load(os.path.join(tmp_path, "rank%d.npz" % q)) for q in range(world)]
    nv = 6
    for q in range(world):
        assert bool(r[q]["ok"])
        other = 1 - q
        # rank q received the other rank's send buffer: arange tagged with the sender
        want = np.arange(r[q]["ro"][-1] * nv, dtype=np.float64) + 1e6 * (other + 1)
        assert np.array_equal(r[q]["recv"], want)
        assert np.array_equal(r[q]["s"], [3.0, 2.0]) and np.array_equal(r[q]["m"], [2.0, 0.0])


def test_thread_comm_allreduce():
    from ocfd_b200.shard import OP_MAX, OP_SUM, ThreadComm
    hub = ThreadComm(3, timeout=30)
    out = [None] * 3

    def run(r):
        c = hub.comm(r)
        out[r] = (c.allreduce(np.array([r, 1.0]), OP_SUM), c.allreduce(np.array([r, -r]), OP_MAX))

    th = [threading.Thread(target=run, args=(r,)) for r in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join(60)
    for r in range(3):
        assert np.array_equal(out[r][0], [3.0, 3.0]) and np.array_equal(out[r][1], [2.0, 0.0])
