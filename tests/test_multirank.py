"""The replica path of bench.py --gpus N on CPU: two gloo ranks combine their device
times (max) and units (sum) exactly as the NCCL ranks do on GPUs, and each rank
gets its own seeded scene."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 10.0 + 5.0 * rank          # rank 1 is the slower one
    units = 1000.0 * (rank + 1)
    out = bench.combine_ranks(ms, units, 2 * ms, 2 * units, dist)
    seed_idx = bench.replica_seed_index(rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out, seed_idx))


def test_two_gloo_ranks_combine_max_time_sum_units():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, (ms, units, e2e_ms, e2e_units), seed_idx in res:
        assert ms == 15.0 and units == 3000.0
        assert e2e_ms == 30.0 and e2e_units == 6000.0
        assert seed_idx == rank
    # whole-job throughput = summed units over the slowest rank's time
    assert res[0][1][1] / (res[0][1][0] / 1e3) == pytest.approx(3000.0 / 0.015)


def test_single_process_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_ranks(1.0, 2.0, 3.0, 4.0, None) == (1.0, 2.0, 3.0, 4.0)
