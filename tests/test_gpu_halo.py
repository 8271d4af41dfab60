"""The Euler/AUSM stage kernels against one another and the oracle: the
halo-staged tile kernel (tile + halo copied into shared memory by bulk
copies), the per-lane tile kernel (the default), the per-cell kernel and the
warp-tiled kernel.

Both kernels evaluate the same face fluxes F(l, r) from the same face states
and sum them in hom3's order; the compiler may still fuse a product into a
sum (FMA) at different places in the two kernels, so their states agree to a
few ulps, step after step (FP64: 1e-13 relative; FP32 face fluxes: 1e-5), on
every grid kind the stage meets: uniform and refined trees (coarse/fine
sub-face groups inside a tile and in its halo), periodic partners, partial
last tiles, batches of grids, every time integration and both precisions,
and any persistent grid size (one block looping over many tiles)."""
import numpy as np
import pytest

import cases
import hom3_b200 as hb
from hom3_b200 import _ffi as F
from oracle import h3o

pytestmark = pytest.mark.gpu


def _pair(o, precision=0):
    """(halo-staged kernel, per-lane tile kernel) solvers from the oracle's state."""
    a = cases.gpu_solver_from_oracle(o, precision)
    b = cases.gpu_solver_from_oracle(o, precision)
    a.set_option(F.OPT_EULER_KERNEL, 0)
    b.set_option(F.OPT_EULER_KERNEL, 1)
    return a, b


TOL = {0: 1e-13, 1: 1e-5}  # FP64, mixed (FP32 face fluxes)


def _same(a, b, fg, what, precision=0):
    from test_gpu_parity import rel_err
    qa, qb = a.state(0)[:, :fg], b.state(0)[:, :fg]
    assert np.isfinite(qa).all(), what
    e = rel_err(qa, qb)
    assert e <= TOL[precision], f"{what}: rel err {e:.3e}"
    assert abs(a.dt() - b.dt()) <= TOL[precision] * b.dt(), what


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
        _same(a, b, fg, f"after {n} more steps", precision)


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


@pytest.mark.parametrize("kernel", [0, 3, 4])
def test_partial_last_tile_and_warp_against_oracle(kernel):
    """A tree whose interior cell count is not a multiple of the tile size
    (256) nor of the warp size (32): the last warp's missing cells include
    ghost indices that must not be taken for cells of the warp."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.3, 0.6, 0.5], 0.2, 5)
    o = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=cases.neumann_cube(w), ic_kind=h3o.IC_SHOCK_TUBE,
                     ic=[0, 0, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1], time_end=1.0, cfl=0.4)
    o.initialize()
    assert o.first_ghost % 32 != 0
    g = cases.gpu_solver_from_oracle(o)
    g.set_option(F.OPT_EULER_KERNEL, kernel)
    assert g.kernel_info()["kernel"] == ("halo", "tile", "cell", "warp", "tile512")[kernel]
    o.solve(1)
    g.solve(1)
    fg = o.first_ghost
    from test_gpu_parity import rel_err
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12
    o.solve(3)
    g.solve(3)
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-10


@pytest.mark.parametrize("kernel", [0, 2, 3, 4])
@pytest.mark.parametrize("precision", [F.FP64, F.MIXED])
def test_stage_kernels_batches(precision, kernel):
    """Batches of grids (a warp's cells never span two grids) in the
    halo-staged (0), per-cell (2) and warp-tiled (3) kernels against the
    per-lane tile kernel."""
    from test_gpu_batch import members
    from hom3_b200.solver import euler_neumann
    ms, tables, states = members(7)
    conds = [[euler_neumann() for _ in range(4)] for _ in tables]

    def make(k):
        b = hb.Batch(2, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, precision, cfl=0.4, time_end=1e9)
        b.set_grids(tables, conds)
        b.set_state(np.concatenate(states, axis=1), 0)
        b.reset_time()
        b.set_option(F.OPT_EULER_KERNEL, k)
        return b

    a, b = make(kernel), make(1)
    a.solve(6)
    b.solve(6)
    from test_gpu_parity import rel_err
    assert rel_err(a.state(0), b.state(0)) <= TOL[0 if precision == F.FP64 else 1]
    assert np.array_equal(a.instances()[2], b.instances()[2])


@pytest.mark.parametrize("slots", [32, 64])
def test_halo_entries_beyond_shared_memory_read_from_global(slots):
    """With fewer shared-memory halo slots than a tile's halo, the remaining
    entries' face states are computed from global memory where a face reads
    them: the same results."""
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    a, b = _pair(o)
    a.set_option(F.OPT_HALO_SLOTS, slots)
    info = a.kernel_info()
    assert info["halo_slots"] == slots and info["max_halo"] > slots
    a.solve(4)
    b.solve(4)
    _same(a, b, o.first_ghost, f"{slots} slots")


@pytest.mark.parametrize("kernel", [2, 3, 4])
@pytest.mark.parametrize("case", ["refined_rk2", "refined_fe_mixed", "explosion_rk3", "periodic_vortex"])
def test_per_cell_and_warp_ausm_kernels(case, kernel):
    """The per-cell AUSM kernel (2: each face from both sides, no shared
    memory), the warp-tiled one (3: face states once per warp, each face
    inside a warp once) and the per-lane kernel on 512-cell tiles (4; 3D
    grids, the 256-cell tiles in 2D) against the per-lane tile kernel and the
    oracle."""
    precision = 1 if case.endswith("mixed") else 0
    if case.startswith("refined"):
        _, (o,) = cases.refined_case(ti=h3o.RK2 if "rk2" in case else h3o.EULER_FORWARD, level=3, fine=5)
    elif case == "explosion_rk3":
        _, (o,) = cases.euler_case("explosion", nd=3, level=4, ti=h3o.SSPRK3)
    else:
        _, (o,) = cases.periodic_vortex_case(level=6, ti=h3o.RK2)
    a, b = _pair(o, precision)
    a.set_option(F.OPT_EULER_KERNEL, kernel)
    want = {2: "cell", 3: "warp", 4: "tile512" if case != "periodic_vortex" else "tile"}[kernel]
    assert a.kernel_info()["kernel"] == want
    fg = o.first_ghost
    o.solve(1)
    a.solve(1)
    b.solve(1)
    _same(a, b, fg, "1 step", precision)
    if precision == 0:
        from test_gpu_parity import rel_err
        assert rel_err(a.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12
    a.solve(5)
    b.solve(5)
    _same(a, b, fg, "6 steps", precision)
