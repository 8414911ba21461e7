"""Host-side logic of the batched engine and the learned path, on the CPU: the Philox
restatement against the generator's published known answers, the grid choice, element classes,
the autocorrelation-time estimate, and the split of boxes over GPUs (gloo, world size 2)."""

import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from epsr_python_translation_b200.batch import choose_grid, element_class, partition_boxes
from epsr_python_translation_b200.learned import integrated_time
from oracle.batch_ref import philox


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors (Random123's published test vectors)."""
    assert philox((0, 0, 0, 0), 0, 0) == (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)
    assert philox((0xffffffff,) * 4, 0xffffffff, 0xffffffff) == (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)
    assert philox((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), 0xa4093822, 0x299f31d0) == \
        (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)


@pytest.mark.parametrize("R", [0.05, 0.1, 0.17, 0.22, 0.3, 0.45, 0.6])
def test_grid_choice_is_valid_and_maximal(R):
    g = choose_grid(R, 0.005)
    assert g is not None
    s, n = g
    assert n % s == 0 and (s - 1) / n >= R
    best = max(((n2 // s2) ** 3 for s2 in range(2, 9) for n2 in range(s2, 200, s2) if (s2 - 1) / n2 >= R),
               default=0)
    assert (n // s) ** 3 == best


def test_element_classes():
    assert [element_class(x) for x in ("S", "Si", "OD", "OW", "O", "C", "HC", "HW", "N", "X")] == \
        [0, 0, 2, 2, 2, 1, 3, 3, 1, 1]


def test_integrated_time_of_ar1():
    rng = np.random.default_rng(1)
    phi = 0.8
    n = 200000
    x = np.zeros(n)
    e = rng.standard_normal(n)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    tau = integrated_time(x)
    assert abs(tau - (1 + phi) / (1 - phi)) < 0.15 * (1 + phi) / (1 - phi)
    assert integrated_time(rng.standard_normal(10000)) < 1.3


def _rank(rank, world, natoms, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    parts = partition_boxes(natoms, world)
    mine = parts[rank]
    import torch
    t = torch.zeros(len(natoms), dtype=torch.int64)
    t[mine] = 1
    dist.all_reduce(t)
    load = torch.tensor([sum(natoms[i] for i in mine)], dtype=torch.int64)
    loads = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(loads, load)
    if rank == 0:
        out.put((t.tolist(), [int(x.item()) for x in loads]))
    dist.destroy_process_group()


def test_boxes_split_over_two_ranks_cover_every_box_once():
    rng = np.random.default_rng(1)
    natoms = [int(x) for x in np.exp(rng.uniform(np.log(300), np.log(30000), 64))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, natoms, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    cover, loads = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert cover == [1] * 64
    assert sum(loads) == sum(natoms)
    assert max(loads) - min(loads) <= max(natoms)
