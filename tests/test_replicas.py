"""Multi-GPU form of the step: replicas only (the domain never shards), so the
only cross-rank operation is the max of the ranks' device times. Tested here
with world size 2 on the gloo backend (CPU); each rank also steps its own
oracle replica to show ranks share no state."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import datetime

    import numpy as np
    import torch.distributed as dist

    import bench
    import pyoracle
    from fortran_loadfile_mitiwing_b200 import cases
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    case = cases.small_case(n_steps=20, seed=100 + rank)
    o = pyoracle.Oracle.from_case(case)
    rows = o.run(5)
    local_ms = 10.0 * (rank + 1)
    value, tmax = bench.replica_value(local_ms, case.params.nx * case.params.ny, 5, world, device="cpu")
    out[rank] = (value, tmax, float(np.abs(rows[:, 1]).sum()))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_value_takes_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (v0, t0, c0), (v1, t1, c1) = out[0], out[1]
    assert t0 == t1 == 20.0
    assert v0 == v1 == pytest.approx(96 * 64 * 5 * 2 / 0.020 / 1e6)
    assert c0 != c1   # different seeds: independent replicas


def test_single_rank_value():
    sys.path.insert(0, ROOT)
    import bench
    v, t = bench.replica_value(4.0, 1000, 10, 1, device="cpu")
    assert t == 4.0 and v == pytest.approx(1000 * 10 / 0.004 / 1e6)
