"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

The oracle builds hom3's grid and initial state; its hom3-numbered tables and
state go through h3c_set_grid / h3c_set_state exactly as a hom3 Solver would
hand them over, and both sides then step.  Tolerances: FP64 path <= 1e-12
relative per step (the bar this path is held to), multi-step runs <= 1e-10 (rounding of
FMA-contracted kernels against the oracle's uncontracted arithmetic compounds
over steps); mixed path (FP32 face fluxes) <= 1e-5 relative per step.
"""
import numpy as np
import pytest

import cases
from oracle import h3o

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-12
TOL_MULTI = 1e-10


def rel_err(a, b):
    """max over variables of max|a - b| / scale_v, scale_v = max|b_v| floored at
    1e-6 of the largest variable (a variable that is analytically zero, e.g. the
    transverse momentum of a 1D problem, carries only rounding noise)."""
    big = max(np.abs(b).max(), 1e-300)
    r = 0.0
    for v in range(b.shape[0]):
        scale = max(np.abs(b[v]).max(), 1e-6 * big)
        r = max(r, np.abs(a[v] - b[v]).max() / scale)
    return r


def check_pair(o, g, tol, what=""):
    fg = o.first_ghost
    qo, qg = o.state(0)[:, :fg], g.state(0)[:, :fg]
    assert np.isfinite(qg).all(), what
    e = rel_err(qg, qo)
    assert e <= tol, f"{what}: rel err {e:.3e} > {tol:.1e}"
    assert abs(g.dt() - o.dt()) <= tol * abs(o.dt()) + 1e-300, (what, g.dt(), o.dt())
    assert abs(g.time() - o.time()) <= tol * max(abs(o.time()), 1e-300) + 1e-300, (what, g.time(), o.time())
    assert g.step() == o.step()
    return e


def run_single(o, nsteps=(1, 4), precision=0, tol_step=TOL_STEP, tol_multi=TOL_MULTI):
    g = cases.gpu_solver_from_oracle(o, precision)
    assert abs(g.dt() - o.dt()) <= tol_step * o.dt()  # initialize()'s set_dt
    o.solve(nsteps[0])
    g.solve(nsteps[0])
    check_pair(o, g, tol_step, "first step")
    o.solve(nsteps[1])
    g.solve(nsteps[1])
    return check_pair(o, g, tol_multi, f"after {sum(nsteps)} steps")


@pytest.mark.parametrize("name", ["constant", "sod", "p123", "explosion"])
@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_euler_3d(name, ti):
    _, (o,) = cases.euler_case(name, nd=3, level=4, ti=ti)
    run_single(o)


@pytest.mark.parametrize("flux", [h3o.AUSM, h3o.LLF])
@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_euler_vortex_2d(flux, ti):
    _, (o,) = cases.euler_case("vortex", level=6, ti=ti, flux=flux)
    run_single(o)


def test_euler_llf_sod_3d():
    _, (o,) = cases.euler_case("sod", nd=3, level=4, flux=h3o.LLF)
    run_single(o)


@pytest.mark.parametrize("nd", [2, 3])
def test_euler_dirichlet_neumann_flux(nd):
    _, (o,) = cases.euler_dirichlet_case(nd=nd, level=5 if nd == 2 else 4)
    run_single(o)


def test_euler_constant_state_preserved():
    """euler_fv_solver_test.cpp:82-112: the solution is the initial condition for all t."""
    _, (o,) = cases.euler_case("constant", nd=3, level=4)
    g = cases.gpu_solver_from_oracle(o)
    q0 = g.state(0)[:, : o.first_ghost]
    g.solve(10)
    assert np.array_equal(g.state(0)[:, : o.first_ghost], q0)


@pytest.mark.parametrize("name", ["constant", "sod", "walls", "slip", "isothermal"])
@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_cns_2d(name, ti):
    _, (o,) = cases.cns_case(name, level=5, ti=ti)
    run_single(o, nsteps=(1, 3))


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_heat_3d(ti):
    _, (o,) = cases.heat_case(level=3, ti=ti)
    run_single(o, nsteps=(1, 6))


def test_mixed_precision_euler():
    _, (o,) = cases.euler_case("sod", nd=3, level=4, ti=h3o.RK2)
    run_single(o, precision=1, tol_step=1e-5, tol_multi=1e-4)


def _coupled(solvers, couple):
    import hom3_b200 as hb
    gs = [cases.gpu_solver_from_oracle(o) for o in solvers]
    for o, g, other in zip(solvers, gs, reversed(gs)):
        g.set_partner(other, o.partner_cells())
    return gs


def test_cht_coupled():
    """coupled_cns_heat_test.cpp:235-248: coupling::apply, cns.solve, heat.solve."""
    import hom3_b200 as hb
    _, (cns, heat) = cases.cht_case(level=7)
    gc, gh = _coupled([cns, heat], None)
    for it in range(3):
        h3o.couple_cht(cns, heat, 0.01)
        hb.couple_cht(0.01, gc, gh)
        cns.solve(); gc.solve()
        heat.solve(); gh.solve()
        check_pair(cns, gc, TOL_STEP if it == 0 else TOL_MULTI, f"cns step {it}")
        check_pair(heat, gh, TOL_STEP if it == 0 else TOL_MULTI, f"heat step {it}")


@pytest.mark.parametrize("kappa", [0.0, 10.0])
def test_cht_hot_solid_conductivity_ratio(kappa):
    """A solid hotter than the flow (heat flows through the interface);
    EXTENSION: conductivity ratio kappa = 10 in the interface temperature."""
    import hom3_b200 as hb
    _, (cns, heat) = cases.cht_case(level=7, kappa=kappa, heat_T=1.3)
    gc, gh = _coupled([cns, heat], None)
    for it in range(4):
        h3o.couple_cht(cns, heat, 0.01)
        hb.couple_cht(0.01, gc, gh)
        cns.solve(); gc.solve()
        heat.solve(); gh.solve()
        check_pair(cns, gc, TOL_STEP if it == 0 else TOL_MULTI, f"cns step {it}")
        check_pair(heat, gh, TOL_STEP if it == 0 else TOL_MULTI, f"heat step {it}")


def test_cht_solve_graph_matches_per_call_loop():
    """h3c_cht_solve (coupled steps replayed from one CUDA graph) equals the
    per-call loop coupling::apply, cns.solve, heat.solve, and the oracle."""
    import hom3_b200 as hb
    _, (cns, heat) = cases.cht_case(level=7, kappa=10.0, heat_T=1.3)
    ga, ha = _coupled([cns, heat], None)
    gb, hb_ = _coupled([cns, heat], None)
    hb.cht_solve(0.01, ga, ha, 19)
    for _ in range(19):
        hb.couple_cht(0.01, gb, hb_)
        gb.solve(1)
        hb_.solve(1)
        h3o.couple_cht(cns, heat, 0.01)
        cns.solve()
        heat.solve()
    for x, y, o in ((ga, gb, cns), (ha, hb_, heat)):
        fg = o.first_ghost
        assert np.array_equal(x.state(0)[:, :fg], y.state(0)[:, :fg])
        check_pair(o, x, TOL_MULTI, "cht_solve vs oracle")


def test_euler_euler_coupled():
    """coupled_euler_euler_test.cpp:155-162."""
    import hom3_b200 as hb
    _, (a, b) = cases.euler_euler_case(level=4)
    ga, gb = _coupled([a, b], None)
    for it in range(3):
        h3o.couple_equal(a, b)
        hb.couple_equal(ga, gb)
        a.solve(); ga.solve()
        b.solve(); gb.solve()
        check_pair(a, ga, TOL_STEP if it == 0 else TOL_MULTI, f"s0 step {it}")
        check_pair(b, gb, TOL_STEP if it == 0 else TOL_MULTI, f"s1 step {it}")


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_refined_tree_extension(ti):
    """EXTENSION (not in hom3): coarse/fine faces on a 2:1 balanced tree."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 5)
    o = w.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=cases.neumann_cube(w), ic_kind=h3o.IC_SHOCK_TUBE,
                     ic=[0, 0, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1], time_end=1.0, cfl=0.4)
    o.initialize()
    run_single(o)


def test_device_order_is_morton_identity_for_minlevel():
    """A MinLevel grid's hom3 leaf order is already the Morton order."""
    _, (o,) = cases.euler_case("sod", nd=3, level=3)
    g = cases.gpu_solver_from_oracle(o)
    perm = g.device_order()
    assert np.array_equal(perm, np.arange(o.ncells))


def test_invalid_tables_rejected():
    import hom3_b200 as hb
    _, (o,) = cases.euler_case("sod", nd=2, level=3)
    t = o.tables()
    s = hb.Solver(2)
    nb = t["neighbors"].copy()
    nb[0, 5] = -7  # an internal cell without neighbour
    with pytest.raises(hb.H3cError):
        s.set_grid(nb, t["x_center"], t["length"], t["bc_idx"], t["first_ghost"], [])


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
@pytest.mark.parametrize("flux", [h3o.AUSM, h3o.LLF])
def test_tile_kernel_matches_per_cell_kernel(ti, flux):
    """The shared-memory tile kernel shares each same-level face flux between
    its two cells (hom3 evaluates the same F(l, r) twice); it must agree with
    the per-cell kernel to rounding (FMA contraction may differ at the point
    where a flux is stored versus consumed in registers)."""
    from hom3_b200 import _ffi as F
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 5)
    o = w.add_solver(h3o.EULER, flux, ti, bcs=cases.neumann_cube(w), ic_kind=h3o.IC_EXPLOSION,
                     ic=[0.5, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1], time_end=1.0, cfl=0.4)
    o.initialize()
    a = cases.gpu_solver_from_oracle(o)
    b = cases.gpu_solver_from_oracle(o)
    b.set_option(F.OPT_TILE_KERNEL, 0)
    a.solve(5)
    b.solve(5)
    fg = o.first_ghost
    assert rel_err(a.state(0)[:, :fg], b.state(0)[:, :fg]) <= 1e-13


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3])
def test_graph_replay_matches_single_steps(ti):
    """Runs of steps replay a captured CUDA graph and single steps a one-step
    graph; interleaved odd counts exercise forward Euler's buffer swap against
    the captured pointers.  Against the same steps launched without graphs."""
    from hom3_b200 import _ffi as F
    _, (o,) = cases.euler_case("sod", nd=3, level=4, ti=ti)
    a = cases.gpu_solver_from_oracle(o)
    b = cases.gpu_solver_from_oracle(o)
    b.set_option(F.OPT_GRAPHS, 0)
    for n in (9, 3, 16, 1, 8):
        a.solve(n)
        for _ in range(n):
            b.solve(1)
    fg = o.first_ghost
    assert np.array_equal(a.state(0)[:, :fg], b.state(0)[:, :fg])
    assert a.time() == b.time() and a.step() == b.step() == 37
    o.solve(37)
    assert rel_err(a.state(0)[:, :fg], o.state(0)[:, :fg]) <= TOL_MULTI * 10


def test_newton_reciprocals_within_2ulp():
    """Reciprocal and rsqrt by Newton-Raphson against IEEE division / sqrt."""
    import ctypes as C
    from hom3_b200 import _ffi as F
    rng = np.random.default_rng(0)
    x = np.concatenate([10.0 ** rng.uniform(-12, 12, 200000), rng.uniform(0.5, 2.0, 100000)])
    r = np.empty_like(x)
    rs = np.empty_like(x)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    F.check(F.lib().h3c_selftest_nr(dp(x), x.size, dp(r), dp(rs)))
    ulp = lambda v: np.spacing(np.abs(v))
    assert np.max(np.abs(r - 1.0 / x) / ulp(1.0 / x)) <= 2.0
    ref = 1.0 / np.sqrt(x)
    assert np.max(np.abs(rs - ref) / ulp(ref)) <= 2.0


def test_set_grid_twice_reuses_solver():
    """Re-initialising a solver (a second h3c_set_grid) must leave it usable."""
    _, (o,) = cases.euler_case("sod", nd=3, level=3)
    g = cases.gpu_solver_from_oracle(o)
    g.solve(2)
    g2 = cases.gpu_solver_from_oracle(o)
    t = o.tables()
    from hom3_b200.solver import Condition
    info = o.info()
    g.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"],
               [Condition(k, v) for k, v in info["bcs"]])
    g.set_state(o.state(0), 0)
    g.reset_time()
    g.solve(3)
    g2.solve(3)
    assert np.array_equal(g.state(0), g2.state(0))


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_taylor_green_cns_periodic(ti):
    """EXTENSION: CNS with periodic conditions (Taylor-Green vortex)."""
    _, (o,) = cases.tgv_case(level=4, ti=ti)
    run_single(o, nsteps=(1, 3))


@pytest.mark.parametrize("flux", [h3o.AUSM, h3o.LLF])
def test_periodic_vortex_euler(flux):
    """EXTENSION: periodic 2D isentropic vortex (first benchmark configuration's setup)."""
    _, (o,) = cases.periodic_vortex_case(level=6, flux=flux)
    run_single(o)


# ---- EXTENSION (not in hom3): SSP-RK3 and MUSCL reconstruction ----
MUSCL = dict(recon=h3o.RECON_MUSCL, limiter_k=1.0)


@pytest.mark.parametrize("name", ["sod", "explosion"])
def test_ssprk3_euler_3d(name):
    _, (o,) = cases.euler_case(name, nd=3, level=4, ti=h3o.SSPRK3)
    run_single(o)


def test_ssprk3_heat_and_cns():
    _, (o,) = cases.heat_case(level=3, ti=h3o.SSPRK3)
    run_single(o, nsteps=(1, 6))
    _, (o,) = cases.cns_case("sod", level=5, ti=h3o.SSPRK3)
    run_single(o, nsteps=(1, 3))


@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3])
def test_muscl_periodic_vortex(ti):
    _, (o,) = cases.periodic_vortex_case(level=6, ti=ti, **MUSCL)
    run_single(o, nsteps=(1, 6))


@pytest.mark.parametrize("name", ["sod", "explosion"])
def test_muscl_euler_3d(name):
    _, (o,) = cases.euler_case(name, nd=3, level=4, ti=h3o.SSPRK3, **MUSCL)
    run_single(o)


def test_muscl_dirichlet_neumann():
    _, (o,) = cases.euler_dirichlet_case(nd=2, level=5, ti=h3o.RK2, **MUSCL)
    run_single(o)


@pytest.mark.parametrize("ti", [h3o.RK2, h3o.SSPRK3])
def test_muscl_refined_tree(ti):
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 5)
    o = w.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=cases.neumann_cube(w), ic_kind=h3o.IC_EXPLOSION,
                     ic=[0.5, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1], time_end=1.0, cfl=0.4, **MUSCL)
    o.initialize()
    run_single(o)


def test_muscl_mixed_precision():
    _, (o,) = cases.periodic_vortex_case(level=6, ti=h3o.SSPRK3, **MUSCL)
    run_single(o, precision=1, tol_step=1e-5, tol_multi=1e-4)


def test_muscl_graph_replay_matches_single_steps():
    _, (o,) = cases.periodic_vortex_case(level=5, ti=h3o.SSPRK3, **MUSCL)
    a = cases.gpu_solver_from_oracle(o)
    b = cases.gpu_solver_from_oracle(o)
    a.solve(19)
    for _ in range(19):
        b.solve(1)
    fg = o.first_ghost
    assert np.array_equal(a.state(0)[:, :fg], b.state(0)[:, :fg])


# ---- advection (advection/physics.hpp, advection/boundary_conditions.hpp) ----
def test_advection_hom3_case():
    """advection_fv_solver_test.cpp:51-125 at its own level 7: the disc in the
    rotating field, characteristic conditions, upwind flux, forward Euler, CFL 1."""
    _, (o,) = cases.advection_case(level=7)
    run_single(o)


@pytest.mark.parametrize("bc", [h3o.BC_ADV_DIRICHLET, h3o.BC_ADV_NEUMANN, h3o.BC_PERIODIC])
@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3])
@pytest.mark.parametrize("flux", [h3o.LLF, h3o.UPWIND])
def test_advection_fluxes_and_conditions(flux, ti, bc):
    _, (o,) = cases.advection_case(level=6, flux=flux, ti=ti, bc_kind=bc, cfl=0.4)
    run_single(o)


def test_advection_3d_uniform_velocity():
    _, (o,) = cases.advection_case(level=4, nd=3, flux=h3o.LLF, ti=h3o.RK2, vel_kind=h3o.VEL_CONSTANT,
                                   vel=(0.3, -0.5, 0.7), bc_kind=h3o.BC_ADV_NEUMANN, cfl=0.3)
    run_single(o)


@pytest.mark.parametrize("flux", [h3o.LLF, h3o.UPWIND])
def test_advection_refined_tree(flux):
    """EXTENSION: coarse/fine faces (area-weighted sub-face fluxes)."""
    _, (o,) = cases.advection_case(level=4, fine=6, flux=flux, ti=h3o.RK2, cfl=0.3)
    run_single(o)


def test_advection_graph_replay_and_min_dt():
    """20 steps replayed from the captured graph, and Solver::min_dt."""
    _, (o,) = cases.advection_case(level=6, flux=h3o.LLF, ti=h3o.RK2, cfl=0.4)
    g = cases.gpu_solver_from_oracle(o)
    assert abs(g.min_dt() - o.min_dt()) <= 1e-15 * o.min_dt()
    o.solve(20)
    g.solve(20)
    check_pair(o, g, TOL_MULTI, "20 graph steps")


def test_advection_needs_a_velocity():
    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    _, (o,) = cases.advection_case(level=4)
    info = o.info()
    s = hb.Solver(2, F.ADVECTION, F.FLUX_UPWIND, F.EULER_FORWARD, cfl=1.0)
    t = o.tables()
    from hom3_b200.solver import Condition
    s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"],
               [Condition(k, v) for k, v in info["bcs"]])
    s.set_state(o.state(0), 0)
    with pytest.raises(hb.H3cError, match="velocity"):
        s.solve(1)
    with pytest.raises(hb.H3cError, match="velocity"):
        s.min_dt()
    s.set_velocity(o.velocity())
    s.reset_time()
    s.solve(2)
    o.solve(2)
    check_pair(o, s, TOL_MULTI, "after the velocity")
