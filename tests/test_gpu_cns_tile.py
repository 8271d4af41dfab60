"""The CNS tile kernel (tile + two halo layers staged into shared memory,
slopes computed there) against the per-cell CNS kernel and the oracle.

Both kernels evaluate every face flux F(l, r) -- AUSM plus the three-point
viscous flux on the cells' central slopes -- with the same arithmetic and
sum F(minus) - F(plus) in hom3's order; the compiler may fuse a product into
a sum (FMA) at different places in the two kernels, so their states agree to
a few ulps (FP64: 1e-13 relative, FP32 fluxes: 1e-5): on periodic grids
(ghost slopes from periodic partners), on walls, inflow and outflow (ghost
slopes with the walls' sign rule), in both precisions and every time
integration."""
import numpy as np
import pytest

import cases
from hom3_b200 import _ffi as F
from oracle import h3o
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu


def _pair(o, precision=0):
    a = cases.gpu_solver_from_oracle(o, precision)
    b = cases.gpu_solver_from_oracle(o, precision)
    b.set_option(F.OPT_HALO_KERNEL, 0)
    assert a.kernel_info()["kernel"] == "halo", a.kernel_info()
    assert b.kernel_info()["kernel"] == "per_cell"
    return a, b


TOL = {0: 1e-13, 1: 1e-5}  # FP64, mixed (FP32 face fluxes)


def _same(a, b, fg, what, precision=0):
    qa, qb = a.state(0)[:, :fg], b.state(0)[:, :fg]
    assert np.isfinite(qa).all(), what
    e = rel_err(qa, qb)
    assert e <= TOL[precision], f"{what}: rel err {e:.3e}"
    assert abs(a.dt() - b.dt()) <= TOL[precision] * b.dt(), what


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3])
@pytest.mark.parametrize("precision", [0, 1])
def test_cns_tile_equals_per_cell_taylor_green(ti, precision):
    _, (o,) = cases.tgv_case(level=4, ti=ti)
    a, b = _pair(o, precision)
    for n in (1, 3):
        a.solve(n)
        b.solve(n)
        _same(a, b, o.first_ghost, f"{n} steps", precision)


@pytest.mark.parametrize("name", ["sod", "walls", "slip", "isothermal"])
def test_cns_tile_equals_per_cell_2d_conditions(name):
    _, (o,) = cases.cns_case(name, level=5, ti=h3o.RK2)
    a, b = _pair(o)
    for n in (1, 4):
        a.solve(n)
        b.solve(n)
        _same(a, b, o.first_ghost, f"{name}: {n} steps")


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("grid", [1, 5, 0])
def test_cns_tile_any_persistent_grid(grid, precision):
    """Blocks looping over several tiles: each tile's copies land while (FP32)
    or after (FP64) the previous tile's fluxes run."""
    _, (o,) = cases.tgv_case(level=4, ti=h3o.RK2)
    a, b = _pair(o, precision)
    a.set_persistent_blocks(grid)
    a.solve(3)
    b.solve(3)
    _same(a, b, o.first_ghost, f"grid {grid}", precision)


def test_cns_tile_against_oracle_tgv():
    _, (o,) = cases.tgv_case(level=5, ti=h3o.RK2)
    g = cases.gpu_solver_from_oracle(o)
    assert g.kernel_info()["kernel"] == "halo"
    fg = o.first_ghost
    o.solve(1)
    g.solve(1)
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12
    o.solve(4)
    g.solve(4)
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-10
