"""One grid split over several solvers (hom3_b200/domain.py) on the GPU.

Each subdomain is a solver of its own whose exchange ghosts receive the
neighbouring subdomains' stage inputs before every part of a step
(h3c_solve_stage), with the time step the minimum over the subdomains.  The
split run must equal the one-grid run: the same face fluxes read the same
states, so the states agree to the rounding of the stage kernels' different
tile borders (1e-13 relative in FP64, 1e-5 with FP32 face fluxes) and dt,
time and step are the same.  Several subdomains share one device here (in
one process, or as gloo ranks in several processes): the exchanges are
host-ordered copies, no kernel waits on another subdomain."""
import os
import socket
import sys

import numpy as np
import pytest

import cases
from hom3_b200 import _ffi as F
from hom3_b200 import domain
from oracle import h3o
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = {0: 1e-13, 1: 1e-5}


def _tables(o):
    t = o.tables()
    t["ncells"] = o.ncells
    return t


def _maker(o, precision):
    import hom3_b200 as hb
    info = o.info()
    props = {k: info[k] for k in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")}
    return lambda: hb.Solver(info["nd"], info["physics"], info["flux"], info["ti"], precision, **props)


def _conditions(o):
    from hom3_b200.solver import Condition
    return [Condition(k, v) for k, v in o.info()["bcs"]]


def _compare(o, precision, parts, steps, kernel=None):
    one = cases.gpu_solver_from_oracle(o, precision)
    split = domain.LocalDomains(_tables(o), parts, o.info()["nd"], _maker(o, precision), _conditions(o))
    if kernel is not None:
        one.set_option(F.OPT_EULER_KERNEL, kernel)
        for p in split.parts:
            p.s.set_option(F.OPT_EULER_KERNEL, kernel)
    split.set_state(o.state(0))
    fg = o.first_ghost
    for n in steps:
        one.solve(n)
        split.solve(n)
        e = rel_err(split.state(), one.state(0)[:, :fg])
        assert e <= TOL[precision], (parts, n, e)
        for p in split.parts:
            assert abs(p.s.dt() - one.dt()) <= 1e-14 * one.dt()
            assert abs(p.s.time() - one.time()) <= 1e-13 * one.time()
            assert p.s.step() == one.step()
    return split


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3])
@pytest.mark.parametrize("parts", [2, 3])
def test_split_refined_tree_equals_one_grid(ti, parts):
    _, (o,) = cases.refined_case(ti=ti, level=3, fine=5)
    _compare(o, 0, parts, (1, 2, 4))


@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4])
def test_split_with_every_euler_stage_kernel(kernel):
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    _compare(o, 0, 2, (1, 3), kernel)


def test_split_heat():
    """hom3's heat test grid (Dirichlet and Neumann walls) in three parts."""
    _, (o,) = cases.heat_case(level=4, ti=h3o.RK2)
    _compare(o, 0, 3, (1, 3))


def test_split_mixed_precision():
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    _compare(o, 1, 3, (1, 3))


def test_split_headline_tree_into_four():
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=6)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 8)
    from hom3_b200 import workloads as W
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
    o = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_RIEMANN3D_PERTURBED,
                     ic=W.riemann3d_oracle_ic(W.fourier_modes()), time_end=1e30, cfl=0.4)
    o.initialize()
    assert o.first_ghost == 1448336
    split = _compare(o, 0, 4, (1, 2))
    assert all(p.sub.halo.size > 0 for p in split.parts)


def test_parts_run_in_order_and_block_whole_steps():
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    g = cases.gpu_solver_from_oracle(o, 0)
    assert g.stages() == 2
    with pytest.raises(F.H3cError):
        g.solve_stage(1)
    g.solve_stage(0)
    with pytest.raises(F.H3cError):
        g.solve(1)
    g.solve_stage(1)
    g.solve(1)
    ref = cases.gpu_solver_from_oracle(o, 0)
    ref.solve(2)
    fg = o.first_ghost
    assert np.array_equal(g.state(0)[:, :fg], ref.state(0)[:, :fg]) and g.step() == 2


def test_exchange_ghosts_rejected_where_faces_read_slopes():
    _, (o,) = cases.cns_case("sod", level=4)
    t = _tables(o)
    sub = domain.partition(t, 2, o.info()["nd"])[0]
    with pytest.raises(F.H3cError):
        domain._make(sub, _maker(o, 0), _conditions(o))


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
        d = domain.DomainSolver(_tables(o), 3, _maker(o, 0), _conditions(o), rank, world)
        d.set_state(o.state(0))
        d.solve(3)
        got = [None] * world
        dist.all_gather_object(got, (*d.local_state(), d.s.dt(), d.s.time()))
        if rank == 0:
            full = np.zeros((5, o.first_ghost))
            for cells, q, _, _ in got:
                full[:, cells] = q
            np.savez(out, q=full, dt=np.array([g[2] for g in got]), time=np.array([g[3] for g in got]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_on_one_device_equal_one_grid(tmp_path):
    """Two ranks (processes) share the one GPU; their exchanges go through
    host memory over gloo, so no kernel waits on the other rank."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "ranks.npz")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    one = cases.gpu_solver_from_oracle(o, 0)
    one.solve(3)
    fg = o.first_ghost
    assert rel_err(got["q"], one.state(0)[:, :fg]) <= TOL[0]
    assert np.all(np.abs(got["dt"] - one.dt()) <= 1e-14 * one.dt())
    assert np.all(np.abs(got["time"] - one.time()) <= 1e-13 * one.time())
