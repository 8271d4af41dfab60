"""The halo-staged Euler/AUSM stage kernel (tile + halo copied into shared
memory by bulk copies) against the per-lane tile kernel and the oracle.

Both kernels evaluate the same face fluxes F(l, r) with the same arithmetic
and sum them in hom3's order, so their states must be bit-identical, step
after step, on every grid kind the stage meets: uniform and refined trees
(coarse/fine sub-face groups inside a tile and in its halo), periodic
partners, partial last tiles, batches of grids, every time integration and
both precisions, and any persistent grid size (one block looping over many
tiles, so the copies of the next tile overlap the current one's fluxes)."""
import numpy as np
import pytest

import cases
import hom3_b200 as hb
from hom3_b200 import _ffi as F
from oracle import h3o

pytestmark = pytest.mark.gpu


def _pair(o, precision=0):
    a = cases.gpu_solver_from_oracle(o, precision)
    b = cases.gpu_solver_from_oracle(o, precision)
    b.set_option(F.OPT_HALO_KERNEL, 0)
    return a, b


def _same(a, b, fg, what):
    qa, qb = a.state(0)[:, :fg], b.state(0)[:, :fg]
    assert np.isfinite(qa).all(), what
    assert np.array_equal(qa, qb), f"{what}: max diff {np.max(np.abs(qa - qb)):.3e}"
    assert a.dt() == b.dt() and a.time() == b.time(), what


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3])
@pytest.mark.parametrize("precision", [0, 1])
def test_halo_kernel_equals_tile_kernel_refined(ti, precision):
    _, (o,) = cases.refined_case(ti=ti, level=3, fine=5)
    a, b = _pair(o, precision)
    assert a.kernel_info()["halo"] == 1 and b.kernel_info()["halo"] == 0
    fg = o.first_ghost
    for n in (1, 2, 9):
        a.solve(n)
        b.solve(n)
        _same(a, b, fg, f"after {n} more steps")


@pytest.mark.parametrize("grid", [1, 3, 148, 0])
def test_halo_kernel_any_persistent_grid(grid):
    """grid blocks take the tiles round-robin; 0 is the default (blocks per SM x SMs)."""
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    a, b = _pair(o)
    a.set_persistent_blocks(grid)
    a.solve(3)
    b.solve(3)
    _same(a, b, o.first_ghost, f"grid {grid}")


@pytest.mark.parametrize("nd,level", [(2, 6), (3, 4)])
def test_halo_kernel_uniform_and_periodic(nd, level):
    if nd == 2:
        _, (o,) = cases.periodic_vortex_case(level=level, ti=h3o.RK2)
    else:
        _, (o,) = cases.euler_case("explosion", nd=3, level=level, ti=h3o.RK2)
    a, b = _pair(o)
    a.solve(4)
    b.solve(4)
    _same(a, b, o.first_ghost, "4 steps")


def test_halo_kernel_partial_last_tile_against_oracle():
    """A tree whose interior cell count is not a multiple of the tile size."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.3, 0.6, 0.5], 0.2, 5)
    o = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=cases.neumann_cube(w), ic_kind=h3o.IC_SHOCK_TUBE,
                     ic=[0, 0, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1], time_end=1.0, cfl=0.4)
    o.initialize()
    assert o.first_ghost % 256 != 0
    g = cases.gpu_solver_from_oracle(o)
    assert g.kernel_info()["halo"] == 1
    o.solve(1)
    g.solve(1)
    fg = o.first_ghost
    from test_gpu_parity import rel_err
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12
    o.solve(3)
    g.solve(3)
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-10


@pytest.mark.parametrize("precision", [F.FP64, F.MIXED])
def test_halo_kernel_batches(precision):
    from test_gpu_batch import members
    from hom3_b200.solver import euler_neumann
    ms, tables, states = members(7)
    conds = [[euler_neumann() for _ in range(4)] for _ in tables]

    def make(halo):
        b = hb.Batch(2, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, precision, cfl=0.4, time_end=1e9)
        b.set_grids(tables, conds)
        b.set_state(np.concatenate(states, axis=1), 0)
        b.reset_time()
        b.set_option(F.OPT_HALO_KERNEL, halo)
        return b

    a, b = make(1), make(0)
    a.solve(6)
    b.solve(6)
    assert np.array_equal(a.state(0), b.state(0))
    for x, y in zip(a.instances(), b.instances()):
        assert np.array_equal(x, y)
