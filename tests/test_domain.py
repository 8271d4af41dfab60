"""One grid split over several ranks (hom3_b200/domain.py), on CPU.

The partition cuts the interior cells along the Morton order; each
subdomain's exchange ghosts stand for the cells of other subdomains its
faces read, and before every stage each rank receives their current values.
Here the host logic is checked without a GPU: the tables of every subdomain
(each interior cell reads only local cells, ghosts or exchange ghosts; every
interior cell is owned exactly once), the exchange lists, and -- with two
gloo ranks as child processes -- a stepped stencil (a test stand-in for the
stage kernels that reads every face neighbour and coarse/fine group the way
the kernels do) whose split run equals the one-grid run bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NSTAGES = 3


def tree_tables(level=3, fine=5):
    """A refined 3D tree (coarse/fine sub-face groups) from the oracle's grid layer."""
    from oracle import h3o
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=level)
    w.refine_sphere([0.45, 0.55, 0.5], 0.3, fine)
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
    s = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_SHOCK_TUBE,
                     ic=[0, 0, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1], time_end=1.0, cfl=0.4)
    s.initialize()
    t = s.tables()
    t["ncells"] = s.ncells
    return t


def stencil_stage(q, t, nd=3):
    """A stand-in for one stage on a grid's tables: physical ghosts take their
    boundary cell's value, exchange ghosts (bc index past the physical
    conditions) keep theirs, and every interior cell moves towards the mean of
    what its faces read (a cell, or the mean of a coarse/fine group)."""
    n, fg = int(t["ncells"]), int(t["first_ghost"])
    nb, sub = t["neighbors"], t["subface_cells"]
    nsub = 0 if sub is None else sub.shape[1]
    q = q.copy()
    nphys = t.get("_nphys")
    for g in range(fg, n):
        if nphys is not None and t["bc_idx"][g] >= nphys:
            continue
        links = [v for v in nb[:, g] if 0 <= v < n]
        q[g] = q[links[0]]
    out = q[:fg].copy()
    for p in range(2 * nd):
        v = nb[p, :fg]
        val = np.empty(fg)
        c = (v >= 0) & (v < n)
        val[c] = q[v[c]]
        gmask = (v <= -2) & (-v - 2 < nsub)
        if gmask.any():
            k = -v[gmask] - 2
            acc = q[sub[0, k]].copy()
            for j in range(1, sub.shape[0]):
                acc = acc + q[sub[j, k]]
            val[gmask] = acc / sub.shape[0]
        out = out + 0.05 * (val - q[:fg])
    q[:fg] = out
    return q


def initial(n):
    return np.sin(np.arange(n) * 0.37) + 2.0


def test_partition_covers_every_cell_once_and_reads_only_local_cells():
    from hom3_b200 import domain
    t = tree_tables()
    fg, n = int(t["first_ghost"]), int(t["ncells"])
    assert t["subface_cells"] is not None and t["subface_cells"].shape[1] > 0
    for parts in (1, 2, 3, 5):
        subs = domain.partition(t, parts, 3)
        owned = np.concatenate([s.cells for s in subs])
        assert np.array_equal(np.sort(owned), np.arange(fg))
        sizes = [s.cells.size for s in subs]
        assert max(sizes) - min(sizes) <= 1
        for s in subs:
            lt = s.tables
            nl, fl = lt["ncells"], lt["first_ghost"]
            lnb = lt["neighbors"]
            gid = s.global_ids()
            assert gid.size == nl and fl == s.cells.size
            nsub = 0 if lt["subface_cells"] is None else lt["subface_cells"].shape[1]
            for p in range(6):
                v = lnb[p, :fl]
                plain = (v >= 0) & (v < nl)
                grp = (v <= -2) & (-v - 2 < nsub)
                assert (plain | grp).all()  # every face of an interior cell reads something local
                # the same cell (or the same group's cells) as in the one grid
                assert np.array_equal(gid[v[plain]], t["neighbors"][p, s.cells[plain]])
                if grp.any():
                    gk = -t["neighbors"][p, s.cells[grp]] - 2
                    lk = -v[grp] - 2
                    assert np.array_equal(gid[lt["subface_cells"][:, lk]], t["subface_cells"][:, gk])
            # every ghost (physical or exchange) has exactly one link, to a local interior cell
            for g in range(fl, nl):
                links = [x for x in lnb[:, g] if 0 <= x < nl]
                assert len(links) == 1 and links[0] < fl
            # physical ghosts keep their condition (renumbered in order), exchange ghosts come last
            nphys = s.ghosts.size
            assert np.array_equal(np.asarray(s.conditions)[lt["bc_idx"][fl:fl + nphys]], t["bc_idx"][s.ghosts])
            assert (lt["bc_idx"][fl + nphys:] == len(s.conditions)).all()
            assert np.all(np.diff(lt["bc_idx"][fl:]) >= 0)  # bc-sorted ghosts, as hom3 sorts them
            assert not np.isin(s.halo, s.cells).any()
        # the exchange lists pair the same global cells
        for s in subs:
            for peer, recv in s.recv.items():
                send = subs[peer].send[s.rank]
                assert np.array_equal(subs[peer].cells[send], s.global_ids()[recv])
            assert sorted(s.recv) == sorted(r.rank for r in subs if s.rank in r.send)
        halo_total = sum(s.halo.size for s in subs)
        assert halo_total == sum(v.size for s in subs for v in s.send.values())


def test_morton_keys_order_by_lower_corner():
    from hom3_b200 import domain
    # 2x2 uniform cells: Morton order (x lowest bit) is (0,0), (1,0), (0,1), (1,1)
    xc = np.array([[0.75, 0.25, 0.75, 0.25], [0.75, 0.75, 0.25, 0.25]])
    ln = np.full(4, 0.5)
    k = domain.morton_keys(xc, ln, 4, 2)
    assert list(np.argsort(k)) == [3, 2, 1, 0]


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from hom3_b200 import domain
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = tree_tables()
        subs = domain.partition(t, world, 3)
        me = subs[rank]
        lt = dict(me.tables, _nphys=len(me.conditions))
        q = initial(int(t["ncells"]))[me.global_ids()]
        send = {p: torch.as_tensor(i) for p, i in me.send.items()}
        recv = {p: torch.as_tensor(i) for p, i in me.recv.items()}
        # the time-step minimum: every rank proposes its own, all take the smallest
        slot = torch.tensor([1000 + rank], dtype=torch.int64)
        domain.min_all(slot)
        for _ in range(NSTAGES):
            view = torch.from_numpy(q.reshape(1, -1))
            domain.exchange(view, send, recv)
            q = stencil_stage(view.numpy().reshape(-1), lt)
        got = [None] * world
        dist.all_gather_object(got, (me.cells, q[:me.cells.size], int(slot[0])))
        if rank == 0:
            fg = int(t["first_ghost"])
            full = np.zeros(fg)
            for cells, vals, _ in got:
                full[cells] = vals
            np.savez(out, q=full, slots=np.array([g[2] for g in got]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_split_stages_equal_one_grid(tmp_path, world):
    import torch.multiprocessing as mp
    out = str(tmp_path / "split.npz")
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    split = np.load(out)
    t = tree_tables()
    q = initial(int(t["ncells"]))
    for _ in range(NSTAGES):
        q = stencil_stage(q, t)
    assert np.array_equal(split["q"], q[:int(t["first_ghost"])])
    assert (split["slots"] == 1000).all()
