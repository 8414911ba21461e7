"""Host logic of bench.py's multi-rank path, on CPU with gloo (world size 2): every box
of every rank gets its own ran1 stream, the timing taken is the slowest rank's, and the
reference arm's non-zero ranks return without work."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 20.0, 1: 20.0}


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


@pytest.mark.parametrize("world,boxes", [(1, 16), (2, 16), (8, 4)])
def test_box_seeds_distinct_over_ranks(world, boxes):
    seeds = [bench.box_seed(rank, boxes, r) for rank in range(world) for r in range(boxes)]
    assert len(set(seeds)) == world * boxes and all(s < 0 for s in seeds)


def test_reference_arm_other_ranks_do_nothing(monkeypatch):
    monkeypatch.setenv("RANK", "1")

    class A:
        steps, warmup, config, gpus = 1, 0, "c1_water", 2
    assert bench.reference_arm(A()) == 0
