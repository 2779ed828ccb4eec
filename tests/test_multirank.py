"""The N > 1 path on CPU: world_size-2 gloo ranks running independent replica solves (the
oracle stands in for the device solve), the max-over-ranks timing and the whole-job rate."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import sys
    for p in (os.path.join(ROOT, "opencfd-ec_b200"), os.path.join(ROOT, "oracle"), ROOT):
        sys.path.insert(0, p)
    import datetime
    import time

    import torch.distributed as dist

    import bench
    import oracle_py
    from ocfd_b200 import cases
    os.environ["OCFD_ORACLE_THREADS"] = "1"
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    p, case = cases.config1(scale=0.25, aoa=bench.rank_aoa(rank))
    o = oracle_py.OracleCase(p, case)
    dist.barrier()
    t0 = time.perf_counter()
    o.advance(3)
    ms = (time.perf_counter() - t0) * 1e3 + 10.0 * rank   # make the ranks' times differ
    ms_max = bench.max_over_ranks(ms, dist, "cpu")
    rate = bench.aggregate_rate(world, case.ncells * 3, ms_max)
    _, rms = o.residual()
    np.savez(os.path.join(out_dir, "rank%d.npz" % rank), ms=ms, ms_max=ms_max, rate=rate, rms=rms, ncells=case.ncells)
    o.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas(tmp_path, oracle):
    world, port = 2, _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    r = [np.load(os.path.join(tmp_path, "rank%d.npz" % q)) for q in range(world)]
    # every rank sees the slowest rank's time
    assert float(r[0]["ms_max"]) == float(r[1]["ms_max"]) == max(float(r[0]["ms"]), float(r[1]["ms"]))
    assert np.isclose(float(r[0]["rate"]), world * int(r[0]["ncells"]) * 3 / (float(r[0]["ms_max"]) * 1e-3))
    # replicas are independent: each rank's solve equals a single-process solve at its angle
    import bench
    from ocfd_b200 import cases
    for q in range(world):
        p, case = cases.config1(scale=0.25, aoa=bench.rank_aoa(q))
        o = oracle.OracleCase(p, case)
        o.advance(3)
        np.testing.assert_array_equal(o.residual()[1], r[q]["rms"])
        o.close()
    assert not np.array_equal(r[0]["rms"], r[1]["rms"])
