"""Batched uneven systems: one graph launch for many independent boxes, and
their sharding over GPUs by atom count (no collective)."""
import os

import numpy as np
import pytest

from protomol_b200.batch import shard_by_atoms


def batched_sizes(count=96, seed=4):
    # the water counts of the batched configuration (3 atoms per water)
    return [3 * int(n) for n in np.random.default_rng(seed).integers(100, 3001, count)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shards_cover_every_system_once_and_balance_atoms(world):
    sizes = batched_sizes()
    shards = shard_by_atoms(sizes, world)
    flat = sorted(k for s in shards for k in s)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[k] for k in s) for s in shards]
    # greedy longest-first: no rank exceeds the mean by more than one system
    assert max(loads) - sum(loads) / world <= max(sizes)
    assert shards == shard_by_atoms(sizes, world)          # deterministic


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = batched_sizes()
    mine = shard_by_atoms(sizes, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    load = sum(sizes[k] for k in mine)
    loads = [None] * world
    dist.all_gather_object(loads, load)
    if rank == 0:
        out.put((gathered, loads))
    dist.barrier()
    dist.destroy_process_group()


def test_shards_agree_across_gloo_ranks():
    """Two ranks compute their shards independently (the same greedy rule) and
    exchange them: together they hold every system exactly once."""
    import random
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + random.randint(0, 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, loads = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(k for s in gathered for k in s) == list(range(96))
    assert abs(loads[0] - loads[1]) <= max(batched_sizes())


@pytest.mark.gpu
@pytest.mark.parametrize("one_launch", [True, False])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_equals_members_evaluated_alone(precision, one_launch):
    """The batch's results are its members' own, bit for bit: with the
    column-path pair kernels of the members as one persistent launch over
    their (system, chunk) work items (the two largest boxes here take the
    column path; the others their own cell-path kernels), and with one pair
    launch per member."""
    from protomol_b200 import forces as F
    from protomol_b200 import workloads
    from protomol_b200.batch import Batch
    ws = [workloads.water_box_workload(n, 50 + k) for k, n in enumerate([100, 260, 640, 1000, 1700, 2400])]
    batch = Batch(0)
    batch.set_pair_launch(one_launch)
    alone = []
    layouts = []
    for w in ws:
        topo = F.Topology(w.system)
        fs = [F.ForceFactory.make(topo, d, precision) for d in w.forces]
        out = np.zeros((w.system.n_atoms, 3))
        e = F.ScalarStructure()
        F.evaluate_group(topo, fs, w.system.positions, out, e)
        alone.append((out, e))
        layouts.append(topo.pair_layout())
        batch.add(topo, fs, w.system.positions)
    if precision == "mixed":
        assert layouts[-2:] == ["columns", "columns"] and "cells" in layouts
    for call in range(2):                       # capture, then replay
        batch.zero()
        batch.evaluate()
        for (fb, eb), (fa, ea) in zip(batch.results(), alone):
            # fixed-point forces and the same energy records: bitwise
            assert np.array_equal(fb, fa)
            assert eb.lennard_jones == ea.lennard_jones and eb.coulomb == ea.coulomb
            assert np.array_equal(eb.virial_tensor, ea.virial_tensor)
    batch.close()
