"""One grid split over several solvers (subdomains), one per GPU.

hom3 has no domain decomposition (its solver is serial).  This is the plan
for single large grids: the interior cells are cut along their Morton order
into contiguous, equally sized ranges; each subdomain is a grid of its own
whose ghosts are its physical ghosts plus, as H3C_BC_EXCHANGE ghosts, every
cell of a neighbouring subdomain that one of its faces reads (face
neighbours and the fine cells of coarse/fine sub-face groups).  A step runs
by parts (h3c_solve_stage): before part 0 the subdomains take the minimum of
their cell time steps (an integer min over the ordered bits of
h3c_dtmin_device), and before every part each subdomain receives the current
stage input of the cells its exchange ghosts stand for.  The result is the
single-grid step: every face flux reads the same states.

`partition` builds the subdomains on the host (numpy), `DomainSolver` steps
one subdomain and exchanges over torch.distributed (NCCL between GPUs, or
gloo through host memory), `LocalDomains` steps several subdomains in one
process on one device (exchanges are device copies).  First-order fluxes
without cell slopes only (Euler, heat, advection): a CNS or MUSCL face would
read slopes of the neighbouring subdomain's cells, and the library rejects
exchange ghosts there.  Periodic conditions are not split.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _ffi as F
from .solver import Condition


def morton_keys(x_center, length, first_ghost, nd):
    """Morton keys of the interior cells (lower corners in units of the finest
    cell, x in the lowest bit): the order the library's tiles follow."""
    xc = x_center[:, :first_ghost]
    ln = length[:first_ghost]
    lo = xc - 0.5 * ln[None, :]
    xmin = lo.min(axis=1)
    hmin = ln.min()
    ix = np.rint((lo - xmin[:, None]) / hmin).astype(np.uint64)
    key = np.zeros(first_ghost, np.uint64)
    bits = 64 // nd
    for b in range(bits):
        for d in range(nd):
            key |= ((ix[d] >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * nd + d)
    return key


@dataclass
class Subdomain:
    """One part of a split grid.  `cells` are the global interior cells it
    owns (local interior numbering = this order); `ghosts` the global ids of
    its physical ghosts and `halo` those of its exchange ghosts, in local
    ghost order (physical, bc-sorted, then exchange); `tables` the local grid
    in the layout of h3c_grid (keys as `build_tables` returns them);
    `conditions` the global condition indices its physical ghosts use, in
    local order (the exchange condition comes after them); `send[peer]`
    local interior ids whose states peer receives, `recv[peer]` local ghost
    ids that receive peer's `send[self]`, in the same order."""
    rank: int
    cells: np.ndarray
    ghosts: np.ndarray
    halo: np.ndarray
    tables: dict
    conditions: list
    send: dict = field(default_factory=dict)
    recv: dict = field(default_factory=dict)

    def global_ids(self):
        """The global id of every local cell (interior, physical ghosts, exchange ghosts)."""
        return np.concatenate([self.cells, self.ghosts, self.halo])


def partition(tables: dict, nparts: int, nd: int):
    """Split the grid of `tables` (h3c_grid layout, hom3 numbering) into
    `nparts` subdomains of equal interior cell counts along the Morton order."""
    n, fg = int(tables["ncells"]), int(tables["first_ghost"])
    nb = np.asarray(tables["neighbors"], np.int64)
    xc = np.asarray(tables["x_center"], np.float64)
    ln = np.asarray(tables["length"], np.float64)
    bc = np.asarray(tables["bc_idx"], np.int64)
    sub = tables.get("subface_cells")
    sub = None if sub is None else np.asarray(sub, np.int64)
    nsub = 0 if sub is None else sub.shape[1]
    np_ = 2 * nd
    if nparts < 1 or nparts > fg:
        raise ValueError(f"cannot split {fg} cells into {nparts} parts")
    order = np.argsort(morton_keys(xc, ln, fg, nd), kind="stable")
    owner = np.empty(fg, np.int64)
    bounds = [fg * r // nparts for r in range(nparts + 1)]
    for r in range(nparts):
        owner[order[bounds[r]:bounds[r + 1]]] = r

    def is_cell(v):
        return (v >= 0) & (v < n)

    def is_group(v):
        return (v <= -2) & (-v - 2 < nsub)

    subs = []
    g2l = np.full(n, -1, np.int64)
    gmap = np.full(max(nsub, 1), -1, np.int64)
    for r in range(nparts):
        cells = np.sort(order[bounds[r]:bounds[r + 1]])
        nbl = nb[:, cells]                                           # [2nd][|L|]
        gmask = is_group(nbl)
        groups = np.unique(-nbl[gmask] - 2) if nsub else np.zeros(0, np.int64)
        refs = [nbl[is_cell(nbl)]]
        if groups.size:
            refs.append(sub[:, groups].ravel())
        refs = np.unique(np.concatenate(refs))
        ghosts = refs[refs >= fg]
        ghosts = ghosts[np.argsort(bc[ghosts], kind="stable")]     # bc-sorted, as hom3 sorts ghosts
        interior_refs = refs[refs < fg]
        halo = interior_refs[owner[interior_refs] != r]
        conds = sorted(set(int(b) for b in bc[ghosts]))
        cmap = np.full(max(conds, default=0) + 1, -1, np.int64)
        cmap[conds] = np.arange(len(conds))
        loc = np.concatenate([cells, ghosts, halo])
        nl, fl, ngh = loc.size, cells.size, ghosts.size
        g2l[loc] = np.arange(nl)
        if groups.size:
            gmap[groups] = np.arange(groups.size)
        lnb = np.full((np_, nl), -1, np.int64)
        for p in range(np_):
            v = nbl[p]
            out = np.full(fl, -1, np.int64)
            c = is_cell(v)
            out[c] = g2l[v[c]]
            g = is_group(v)
            if g.any():
                out[g] = -2 - gmap[-v[g] - 2]
            lnb[p, :fl] = out
            gv = nb[p, ghosts]
            gc = (gv >= 0) & (gv < fg)
            lnb[p, fl:fl + ngh][gc] = g2l[gv[gc]]
        # an exchange ghost is linked to one local cell that reads it (the ABI's one-neighbour rule for
        # ghosts; the library does not read the link of an exchange ghost)
        linked = np.zeros(nl, bool)
        for p in range(np_):
            v = nbl[p]
            reads, halos = [], []
            c = is_cell(v)
            reads.append(np.nonzero(c)[0])
            halos.append(g2l[v[c]])
            g = np.nonzero(is_group(v))[0]
            for j in range(nsub and sub.shape[0]):
                reads.append(g)
                halos.append(g2l[sub[j, -v[g] - 2]])
            reads, halos = np.concatenate(reads), np.concatenate(halos)
            keep = (halos >= fl + ngh) & ~linked[halos]
            hs, first = np.unique(halos[keep], return_index=True)
            lnb[p ^ 1, hs] = reads[keep][first]
            linked[hs] = True
        assert linked[fl + ngh:].all()
        lsub = None
        if groups.size:
            lsub = g2l[sub[:, groups]]
        lbc = np.full(nl, -1, np.int32)
        lbc[fl:fl + ngh] = cmap[bc[ghosts]]
        lbc[fl + ngh:] = len(conds)
        lt = dict(neighbors=lnb, x_center=np.ascontiguousarray(xc[:, loc]), length=np.ascontiguousarray(ln[loc]),
                  bc_idx=lbc, first_ghost=fl, ncells=nl, subface_cells=lsub)
        subs.append(Subdomain(r, cells, ghosts, halo, lt, conds))
        g2l[loc] = -1
        if groups.size:
            gmap[groups] = -1
    # exchange lists: the cells of r that are exchange ghosts of s
    for s in subs:
        base = s.tables["ncells"] - s.halo.size
        for r in range(nparts):
            if r == s.rank:
                continue
            mine = s.halo[owner[s.halo] == r]
            if mine.size == 0:
                continue
            subs[r].send[s.rank] = np.searchsorted(subs[r].cells, mine)
            s.recv[r] = base + np.searchsorted(s.halo, mine)
    return subs


def _make(sub: Subdomain, make_solver, conditions):
    s = make_solver()
    t = sub.tables
    conds = [conditions[c] for c in sub.conditions] + [Condition(F.BC_EXCHANGE)]
    s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"], conds, t["subface_cells"])
    return s


class _Part:
    """A subdomain's solver and its exchange index lists in the library's internal numbering."""

    def __init__(self, sub: Subdomain, make_solver, conditions):
        import torch
        self.sub = sub
        self.s = _make(sub, make_solver, conditions)
        perm = self.s.device_order()
        self.send = {p: torch.as_tensor(perm[i], device="cuda") for p, i in sub.send.items()}
        self.recv = {p: torch.as_tensor(perm[i], device="cuda") for p, i in sub.recv.items()}
        self.stream = torch.cuda.ExternalStream(self.s.stream())

    def set_global_state(self, q):
        """q: [nv][n] in the global (hom3) numbering; the exchange ghosts get their cells' states too."""
        self.s.set_state(np.ascontiguousarray(q[:, self.sub.global_ids()]), 0)


class LocalDomains:
    """Several subdomains of one grid stepped in one process on one device:
    the exchanges are device copies between the subdomains' buffers, the
    dt minimum a device minimum.  The reference arrangement for testing the
    split; `DomainSolver` is the one-subdomain-per-rank form."""

    def __init__(self, tables, nparts, nd, make_solver, conditions):
        self.subs = partition(tables, nparts, nd)
        self.parts = [_Part(sub, make_solver, conditions) for sub in self.subs]
        self.n = int(tables["ncells"])
        self.fg = int(tables["first_ghost"])

    def set_state(self, q):
        for p in self.parts:
            p.set_global_state(q)
            p.s.reset_time()

    def _sync(self):
        import torch
        torch.cuda.synchronize()

    def _exchange(self, k):
        import torch
        self._sync()
        views = [p.s.stage_input(k) for p in self.parts]
        for dst, pd in enumerate(self.parts):
            for src, idx in pd.recv.items():
                views[dst][:, idx] = views[src][:, self.parts[src].send[dst]]
        torch.cuda.synchronize()

    def _dt_min(self):
        import torch
        self._sync()
        slots = [p.s.dtmin_device() for p in self.parts]
        m = torch.stack([v[0] for v in slots]).min()
        for v in slots:
            v[0] = m
        torch.cuda.synchronize()

    def solve(self, nsteps=1):
        stages = self.parts[0].s.stages()
        for _ in range(nsteps):
            self._dt_min()
            for k in range(stages):
                self._exchange(k)
                for p in self.parts:
                    p.s.solve_stage(k)

    def state(self):
        """The interior state [nv][first_ghost] in the global numbering."""
        nv = self.parts[0].s.nv
        out = np.zeros((nv, self.fg))
        for p in self.parts:
            q = p.s.state(0)
            out[:, p.sub.cells] = q[:, :p.sub.cells.size]
        return out


def exchange(view, send, recv, group=None):
    """One exchange of a split grid over torch.distributed: `view` [nv][ld]
    holds this rank's cells; send[peer] are the columns peer receives,
    recv[peer] the columns that receive peer's send[self] (index tensors on
    view's device).  NCCL moves device buffers; other backends (gloo) move
    host copies.  Every rank posts all its sends and receives, then waits."""
    import torch
    import torch.distributed as dist
    on_device = view.is_cuda and dist.get_backend(group) == "nccl"
    comm = view.device if on_device else torch.device("cpu")
    ops, bufs = [], {}
    for peer, idx in sorted(send.items()):
        ops.append(dist.P2POp(dist.isend, view[:, idx].contiguous().to(comm), peer, group))
    for peer, idx in sorted(recv.items()):
        bufs[peer] = torch.empty((view.shape[0], idx.numel()), dtype=view.dtype, device=comm)
        ops.append(dist.P2POp(dist.irecv, bufs[peer], peer, group))
    if ops:
        if on_device:
            works = dist.batch_isend_irecv(ops)
        else:
            works = [op.op(op.tensor, op.peer, op.group) for op in ops]
        for w in works:
            w.wait()
    for peer, buf in bufs.items():
        view[:, recv[peer]] = buf.to(view.device)


def min_all(slot, group=None):
    """slot (a 1-element int64 tensor) <- its minimum over the ranks of group."""
    import torch.distributed as dist
    on_device = slot.is_cuda and dist.get_backend(group) == "nccl"
    t = slot.clone() if on_device else slot.cpu()
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    slot.copy_(t.to(slot.device))


class DomainSolver:
    """This rank's subdomain of a grid split over the ranks of `group`
    (torch.distributed): NCCL exchanges device buffers directly, other
    backends go through host memory.  Every rank builds the same partition."""

    def __init__(self, tables, nd, make_solver, conditions, rank, world, group=None):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.rank, self.world = rank, world
        subs = partition(tables, world, nd)
        self.part = _Part(subs[rank], make_solver, conditions)
        self.s = self.part.s
        self.sub = subs[rank]
        self.fg = int(tables["first_ghost"])
        self.torch = torch

    def set_state(self, q):
        self.part.set_global_state(q)
        self.s.reset_time()

    def _exchange(self, k):
        torch = self.torch
        with torch.cuda.stream(self.part.stream):
            exchange(self.s.stage_input(k), self.part.send, self.part.recv, self.group)

    def _dt_min(self):
        if self.world == 1:  # one subdomain: its own minimum is the grid's
            return
        torch = self.torch
        with torch.cuda.stream(self.part.stream):
            min_all(self.s.dtmin_device(), self.group)

    def solve(self, nsteps=1):
        stages = self.s.stages()
        for _ in range(nsteps):
            self._dt_min()
            for k in range(stages):
                self._exchange(k)
                self.s.solve_stage(k)

    def local_state(self):
        """(global ids, interior state [nv][cells]) of this rank's cells."""
        q = self.s.state(0)
        return self.sub.cells, q[:, :self.sub.cells.size]
