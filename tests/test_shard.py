"""Sharding independent grids across ranks (hom3_b200/shard.py), on CPU.

The batched workload's instances are independent, so N ranks split them and
step their shares with no collective on the data path; the results are
gathered at the end.  These tests run two gloo ranks as child processes on
the host: each steps its share of a small ensemble with the oracle (the CPU
restatement of hom3 -- the per-rank stepper here, where no GPU exists) and
the gathered per-instance time steps, times and states must be identical to
one rank stepping every instance."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STEPS = 4


def members():
    from hom3_b200 import workloads as W
    return W.ensemble_members(5, seed=11, nmin=12, nmax=36)


def step_member(m, steps=STEPS):
    """One ensemble member (a 2D isentropic vortex in an nx x ny box embedded
    in a square root cell, +1-level patch) stepped with the oracle."""
    from oracle import h3o
    h, nx, ny, level = m["h"], m["nx"], m["ny"], m["level"]
    side = h * 2 ** level
    w = h3o.World(2, [0.0, 0.0], [side, side], level=level)
    (px, py), pr = m["patch"]
    if pr > 0.5 * h:
        w.refine_sphere([px, py], pr, level + 1)
    lx, ly = nx * h, ny * h
    eps = side * 1e-15
    geoms = [h3o.edge([eps, 0], [1, 0]), h3o.edge([lx - eps, 0], [-1, 0]), h3o.edge([0, eps], [0, 1]),
             h3o.edge([0, ly - eps], [0, -1])]
    s = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=[h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in geoms],
                     domain=h3o.square([0.5 * lx, 0.5 * ly], [lx, ly]), domain_kind=2,
                     ic_kind=h3o.IC_VORTEX_PARAM, ic=[m["beta"], m["centre"][0], m["centre"][1], 1.0, 1.0],
                     cfl=0.4, time_end=1e9)
    s.initialize()
    s.solve(steps)
    fg = s.first_ghost
    return {"cells": int(fg), "dt": s.dt(), "time": s.time(), "step": s.step(), "q": s.state(0)[:, :fg].copy()}


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    from hom3_b200 import shard
    from oracle import h3o
    h3o.set_num_threads(1)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = members()
        cells = [m["nx"] * m["ny"] for m in ms]  # size estimate: the boxes' base cells
        assign = shard.partition(cells, world)
        local = [step_member(ms[i]) for i in assign[rank]]
        got = shard.gather(local, assign, rank)
        if rank == 0:
            np.savez(out, assign=np.array([len(a) for a in assign]),
                     **{f"q{i}": r["q"] for i, r in enumerate(got)},
                     dt=np.array([r["dt"] for r in got]), time=np.array([r["time"] for r in got]),
                     step=np.array([r["step"] for r in got]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_partition_is_balanced_deterministic_and_complete():
    from hom3_b200 import shard
    rng = np.random.default_rng(0)
    cells = rng.integers(1000, 300000, size=256).tolist()
    for ws in (1, 2, 3, 8):
        a = shard.partition(cells, ws)
        assert a == shard.partition(cells, ws)
        assert sorted(i for r in a for i in r) == list(range(len(cells)))
        loads = [sum(cells[i] for i in r) for r in a]
        assert max(loads) - min(loads) <= max(cells)
        assert all(r == sorted(r) for r in a)
    assert shard.partition([5, 1, 1], 2) == [[0], [1, 2]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def test_two_gloo_ranks_gather_what_one_rank_computes(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "two.npz")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    two = np.load(out)
    assert list(two["assign"]) != [5, 0] and sum(two["assign"]) == 5  # both ranks had work
    from oracle import h3o
    h3o.set_num_threads(1)
    one = [step_member(m) for m in members()]
    for i, r in enumerate(one):
        assert np.array_equal(two[f"q{i}"], r["q"]), i
        assert two["dt"][i] == r["dt"] and two["time"][i] == r["time"] and two["step"][i] == r["step"] == STEPS
    assert len({round(r["dt"], 15) for r in one}) > 1  # each instance keeps its own time step
