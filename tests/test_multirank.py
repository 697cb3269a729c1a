"""The N-GPU replica path on CPU: two gloo ranks aggregate their timings the
way bench.py does under torchrun (max over ranks, all ranks' work)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "finite-volume-2d-cpp_b200"))
    import replicas
    dist.init_process_group("gloo", rank=rank, world_size=world)
    seconds = [0.5, 2.0][rank]            # rank 1 is the slow one
    mx = replicas.max_over_ranks(seconds, dist)
    thr = replicas.job_throughput(1000.0, seconds, dist)
    dist.barrier()
    out[rank] = (mx, thr)
    dist.destroy_process_group()


def test_two_rank_aggregation():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (2.0, 2 * 1000.0 / 2.0)


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "finite-volume-2d-cpp_b200"))
    import replicas
    assert replicas.max_over_ranks(3.0) == 3.0
    assert replicas.job_throughput(10.0, 2.0) == 5.0
