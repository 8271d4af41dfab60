"""GPU parity at the benchmarked configurations (not only small grids).

* The 3D Euler refined tree the default bench times: 64^3 base on the unit
  cube, +2 levels inside the sphere r = 0.25 (1,448,336 leaf cells, 25,704
  coarse/fine sub-face groups), the perturbed 3D Riemann problem (16 Fourier
  modes, seed 0), zero-gradient outflow, AUSM, RK2.  The oracle builds hom3's
  tree and state; its hom3-numbered tables and state go through the C ABI.
  FP64: <= 1e-12 relative after one step, <= 1e-10 after three, the
  conserved totals (compensated sums of q * volume) equal to the oracle's to
  1e-12; the mixed path (FP32 face fluxes): relative L2 error of the
  conserved state <= 1e-6 against the FP64 oracle after the same steps.
* The 2D isentropic vortex on a 256^2 periodic grid over [0, 10]^2 (beta 5,
  centre (5, 5)) with MUSCL + SSP-RK3 at CFL 0.5.
* The Taylor-Green vortex (CNS, Re 1600, Mach 0.1, Pr 0.71) on 64^3.
"""
import math
import os

import numpy as np
import pytest

import cases
from hom3_b200 import workloads as W
from oracle import h3o
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu

L2_MIXED = 1e-6  # matched-error bar of the mixed path against the FP64 oracle


def l2_rel(a, b):
    """||a - b||_2 / ||b||_2 over the whole conserved state (every variable of
    every cell): the L2 error the mixed path is held to.  A single variable
    that is nearly zero (the momentum of a fluid at rest) carries relative
    errors of the FP32 fluxes' size, which this norm weighs by its share."""
    return float(np.sqrt(((a - b) ** 2).sum() / (b * b).sum()))


def totals(q, vol):
    """Conserved totals sum_c q_v(c) vol(c), compensated (math.fsum)."""
    return np.array([math.fsum(q[v] * vol) for v in range(q.shape[0])])


@pytest.fixture(scope="module")
def headline():
    h3o.set_num_threads(os.cpu_count() or 1)
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=6)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 8)
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
    o = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_RIEMANN3D_PERTURBED,
                     ic=W.riemann3d_oracle_ic(W.fourier_modes()), time_end=1e30, cfl=0.4)
    o.initialize()
    assert o.first_ghost == 1448336
    assert o.tables()["subface_cells"].shape[1] == 25704
    return w, o


def test_headline_tree_fp64_and_mixed_against_oracle(headline):
    _, o = headline
    fg = o.first_ghost
    vol = o.tables()["length"][:fg] ** 3
    g = cases.gpu_solver_from_oracle(o, 0)
    m = cases.gpu_solver_from_oracle(o, 1)
    assert g.kernel_info()["kernel"] == "tile"
    assert abs(g.dt() - o.dt()) <= 1e-12 * o.dt()
    t0 = totals(o.state(0)[:, :fg], vol)
    o.solve(1)
    g.solve(1)
    m.solve(1)
    qo, qg = o.state(0)[:, :fg], g.state(0)[:, :fg]
    assert rel_err(qg, qo) <= 1e-12
    assert abs(g.dt() - o.dt()) <= 1e-12 * o.dt() and abs(g.time() - o.time()) <= 1e-12 * o.time()
    e1 = l2_rel(m.state(0)[:, :fg], qo)
    assert e1 <= L2_MIXED, e1
    o.solve(2)
    g.solve(2)
    m.solve(2)
    qo, qg = o.state(0)[:, :fg], g.state(0)[:, :fg]
    assert rel_err(qg, qo) <= 1e-10
    assert g.step() == o.step() == 3
    to, tg = totals(qo, vol), totals(qg, vol)
    scale = np.abs(t0).max()
    assert np.all(np.abs(tg - to) <= 1e-12 * scale), (tg - to) / scale
    e3 = l2_rel(m.state(0)[:, :fg], qo)
    assert e3 <= L2_MIXED, e3
    assert g.status() == 0 and m.status() == 0


@pytest.mark.parametrize("kernel", [0, 2, 3, 4])
def test_headline_tree_other_stage_kernels_agree(headline, kernel):
    """The halo-staged tile kernel (0), the per-cell kernel (2), the
    warp-tiled kernel (3) and the per-lane kernel on 512-cell tiles (4) on the
    same tree agree with the default per-lane tile kernel to rounding."""
    from hom3_b200 import _ffi as F
    _, o = headline
    fg = o.first_ghost
    a = cases.gpu_solver_from_oracle(o, 0)
    b = cases.gpu_solver_from_oracle(o, 0)
    b.set_option(F.OPT_EULER_KERNEL, kernel)
    assert b.kernel_info()["kernel"] == ("halo", "tile", "cell", "warp", "tile512")[kernel]
    a.solve(2)
    b.solve(2)
    assert rel_err(a.state(0)[:, :fg], b.state(0)[:, :fg]) <= 1e-13


def test_vortex_256_muscl_ssprk3_against_oracle():
    _, (o,) = cases.periodic_vortex_case(level=8, ti=h3o.SSPRK3, recon=h3o.RECON_MUSCL, limiter_k=1.0)
    assert o.first_ghost == 256 * 256
    fg = o.first_ghost
    g = cases.gpu_solver_from_oracle(o, 0)
    m = cases.gpu_solver_from_oracle(o, 1)
    o.solve(1)
    g.solve(1)
    m.solve(1)
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12
    for _ in range(3):
        o.solve(5)
        g.solve(5)
        m.solve(5)
    qo = o.state(0)[:, :fg]
    assert rel_err(g.state(0)[:, :fg], qo) <= 1e-10
    assert l2_rel(m.state(0)[:, :fg], qo) <= L2_MIXED


def test_taylor_green_64_against_oracle():
    h3o.set_num_threads(os.cpu_count() or 1)
    _, (o,) = cases.tgv_case(level=6, ti=h3o.RK2)
    assert o.first_ghost == 64 ** 3
    fg = o.first_ghost
    g = cases.gpu_solver_from_oracle(o, 0)
    m = cases.gpu_solver_from_oracle(o, 1)
    o.solve(1)
    g.solve(1)
    m.solve(1)
    assert rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12
    o.solve(3)
    g.solve(3)
    m.solve(3)
    qo = o.state(0)[:, :fg]
    assert rel_err(g.state(0)[:, :fg], qo) <= 1e-10
    assert l2_rel(m.state(0)[:, :fg], qo) <= L2_MIXED
