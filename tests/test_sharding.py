"""Target-sharded multi-rank host logic on CPU (gloo, world size 2): leaf
ranges tile the leaves, particle ranges tile the sorted slots, the source
broadcast replicates rank 0's inputs and the all_gather reassembles every
rank's sorted slice."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from jaccpot_b200 import sharding, tree, workloads


def test_ranges_tile_leaves_and_particles():
    pos, mass = workloads.clustered(20000, seed=1)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6)
    for world in (1, 2, 3, 8):
        rs = sharding.leaf_ranges(topo.num_leaves, world)
        assert rs[0][0] == 0 and rs[-1][1] == topo.num_leaves
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        pr = [sharding.particle_range(topo, lo, hi) for lo, hi in rs]
        pr = [r for r in pr if r[1] > r[0]]
        assert pr[0][0] == 0 and pr[-1][1] == topo.num_particles
        assert all(a[1] == b[0] for a, b in zip(pr, pr[1:]))


def _worker(rank, world, port, result_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pos, mass = workloads.clustered(5000, seed=3)
        if rank != 0:  # only rank 0 has the real inputs
            pos = np.zeros_like(pos)
            mass = np.zeros_like(mass)
        tp, tm = torch.from_numpy(pos.copy()), torch.from_numpy(mass.copy())
        sharding.replicate_sources(tp, tm)
        topo = tree.build_topology(tp.numpy(), tm.numpy(), leaf_size=16, theta=0.6)
        lo, hi = sharding.leaf_ranges(topo.num_leaves, world)[rank]
        b, e = sharding.particle_range(topo, lo, hi)
        # stand-in for this rank's evaluation: a value that identifies each slot
        idx = torch.arange(b, e, dtype=torch.float64)
        local = torch.stack([idx, 2 * idx, 3 * idx, idx * 0 + rank], dim=1)
        full = sharding.gather_sorted(local, topo)
        ok = torch.equal(full[:, 0], torch.arange(topo.num_particles, dtype=torch.float64))
        ok = ok and torch.equal(full[:, 2], 3 * full[:, 0])
        owners = full[:, 3].numpy()
        ok = ok and set(np.unique(owners)) == set(range(world))
        ok = ok and np.array_equal(tp.numpy(), workloads.clustered(5000, seed=3)[0])
        with open(f"{result_path}.{rank}", "w") as f:
            f.write("ok" if ok else "bad")
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_on_cpu(tmp_path):
    world = 2
    port = 29500 + (os.getpid() % 1000)
    res = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, port, res), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        assert open(f"{res}.{r}").read() == "ok"
