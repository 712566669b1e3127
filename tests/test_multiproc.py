"""Multi-process host logic of the replicas-only multi-GPU mode, on CPU with gloo
(world size 2): each rank gets its own seed, the step time is the max over ranks,
and the whole-job value aggregates all ranks' particles."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup("gloo")
    seed = bench.replica_seed(r)
    ms = bench.allmax(w, 10.0 + 5.0 * r)          # rank 1 is the slow one
    val = bench.aggregate_value(w, 8, 3, ms)
    bench.barrier(w)
    dist.destroy_process_group()
    out.put((r, w, seed, ms, val))


def test_replicas_gloo_world_size_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, s0, m0, v0), (r1, w1, s1, m1, v1) = res
    assert (w0, w1) == (2, 2)
    assert s0 != s1                      # independent boxes
    assert m0 == m1 == 15.0              # max over ranks
    assert v0 == v1 == pytest.approx(2 * 8 ** 3 * 3 / 0.015)


def test_reference_arm_other_ranks_do_nothing(capsys):
    import argparse

    import bench
    args = argparse.Namespace(size="small", steps=1, warmup=3, gpus=2)
    bench.run_reference(args, world=2, rank=1)   # returns at once, prints nothing
    assert capsys.readouterr().out == ""


class _HostGrads:
    """Stands in for a ForceNet's gradient buffer on a CPU-only host."""

    def __init__(self, g):
        self.g = g

    def grads(self):
        return self.g.copy()

    def set_grads(self, g):
        self.g = g.copy()


def _nn_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import numpy as np
    import torch.distributed as dist

    import bench
    from djb200.nn import allreduce_gradients
    bench.dist_setup("gloo")
    net = _HostGrads(np.arange(6, dtype=np.float32) * (rank + 1))
    allreduce_gradients(net)
    dist.destroy_process_group()
    out.put((rank, net.g.tolist()))


def test_nn_gradient_allreduce_gloo_world_size_2():
    """djb_nn_grads -> all_reduce -> djb_nn_set_grads: both replicas end with the mean."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_nn_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [1.5 * i for i in range(6)]
    assert res[0][1] == pytest.approx(expect) and res[1][1] == pytest.approx(expect)
