"""Discrete adjoint (h3c_adjoint) on the GPU, through the C ABI.

J(q0) = <lambda, q_N> with the forward time steps frozen.  The gradient is
checked against (a) the forward-mode dual-number build of the oracle
(directional derivatives, to rounding), (b) central finite differences of the
GPU's own frozen-dt forward map (h3c_solve_dt) in 32 random directions, to
1e-6 relative, and (c) itself under different checkpoint intervals.  The
states are made smooth first (cases.smooth_state) so that no face sits on a
switch of the AUSM flux, where the derivative does not exist.
"""
import numpy as np
import pytest

import cases
from oracle import h3o

pytestmark = pytest.mark.gpu

BUILDERS = {
    "euler2d_fe": lambda: cases.euler_case("sod", nd=2, level=5, ti=h3o.EULER_FORWARD),
    "euler2d_rk2": lambda: cases.euler_case("sod", nd=2, level=5, ti=h3o.RK2),
    "euler3d_rk2": lambda: cases.euler_case("sod", nd=3, level=3, ti=h3o.RK2),
    "euler_dirichlet_rk2": lambda: cases.euler_dirichlet_case(nd=2, level=4, ti=h3o.RK2),
    "heat3d_fe": lambda: cases.heat_case(level=3),
    "heat3d_rk2": lambda: cases.heat_case(level=3, ti=h3o.RK2),
    "periodic_vortex_rk2": lambda: cases.periodic_vortex_case(level=5),
    "refined_fe": lambda: cases.refined_case(ti=h3o.EULER_FORWARD),
    "refined_rk2": lambda: cases.refined_case(ti=h3o.RK2),
    "euler2d_llf_rk2": lambda: cases.euler_case("sod", nd=2, level=5, ti=h3o.RK2, flux=h3o.LLF),
    "euler3d_llf_fe": lambda: cases.euler_case("sod", nd=3, level=3, ti=h3o.EULER_FORWARD, flux=h3o.LLF),
    "refined_llf_rk2": lambda: _refined_llf(),
}


def _refined_llf():
    """The refined tree of cases.refined_case with the LLF flux: its faces are
    evaluated with the evaluating cell's own length, so a coarse/fine face
    enters the coarse and the fine residual with different dissipation."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=2)
    w.refine_sphere([0.5, 0.5, 0.5], 0.3, 4)
    s = w.add_solver(h3o.EULER, h3o.LLF, h3o.RK2, bcs=cases.neumann_cube(w), ic_kind=h3o.IC_SHOCK_TUBE,
                     ic=[0, 0, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1], time_end=1.0, cfl=0.4)
    s.initialize()
    return w, [s]
NSTEPS = 12


def nsteps(name):
    """Steps of a case: hom3's LLF flux (dissipation dx/dt, euler/physics.hpp:262-267) is unstable in 2D and 3D
    (each face relaxes the cell half-way to its neighbour), so its cases stop before the growth shows."""
    return (2 if "refined" in name else 4) if "llf" in name else NSTEPS


def setup(name, seed=0):
    _, (o,) = BUILDERS[name]()
    q1 = cases.smooth_state(o)
    o.set_state(q1)
    g = cases.gpu_solver_from_oracle(o)
    rng = np.random.default_rng(seed)
    lam = np.zeros_like(q1)
    lam[:, :o.first_ghost] = rng.standard_normal((q1.shape[0], o.first_ghost))
    return o, g, q1, lam


def frozen_J(g, q, dts, lam):
    g.set_state(q, 0)
    g.reset_time()
    g.solve_dt(dts)
    return float((g.state(0) * lam).sum())


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_adjoint_matches_dual_oracle(name):
    o, g, q1, lam = setup(name)
    fg = o.first_ghost
    n = nsteps(name)
    grad, dts = g.adjoint(n, lam, every=min(5, n - 1))
    assert np.isfinite(grad).all()
    assert np.all(grad[:, fg:] == 0.0)
    # the forward of the adjoint took the solver's own CFL steps
    for i in range(n):
        o.solve(1)
        assert abs(dts[i] - o.dt()) <= 1e-12 * o.dt(), (i, dts[i], o.dt())
    rng = np.random.default_rng(11)
    for _ in range(3):
        dq = np.zeros_like(q1)
        dq[:, :fg] = rng.standard_normal((q1.shape[0], fg))
        _, (o2,) = BUILDERS[name]()
        ds = h3o.DualSolver(o2)
        ds.set_state(q1, dq)
        ds.solve_dt(dts)
        _, dot = ds.state()
        jvp = (lam[:, :fg] * dot[:, :fg]).sum()
        vjp = (grad[:, :fg] * dq[:, :fg]).sum()
        scale = np.abs(lam[:, :fg] * dot[:, :fg]).sum()
        assert abs(jvp - vjp) <= 1e-11 * scale, (jvp, vjp, scale)


def fd_worst(name, eps, ndir=32):
    """Largest relative gap between <grad, dq> and central differences of the
    GPU frozen-dt map over ndir random directions dq."""
    o, g, q1, lam = setup(name, seed=2)
    fg = o.first_ghost
    grad, dts = g.adjoint(nsteps(name), lam, every=min(4, nsteps(name) - 1))
    assert np.isfinite(grad).all()
    rng = np.random.default_rng(2)
    worst = 0.0
    for _ in range(ndir):
        dq = np.zeros_like(q1)
        dq[:, :fg] = rng.standard_normal((q1.shape[0], fg))
        fd = (frozen_J(g, q1 + eps * dq, dts, lam) - frozen_J(g, q1 - eps * dq, dts, lam)) / (2 * eps)
        ad = (grad * dq).sum()
        scale = np.abs(grad * dq).sum()
        gap = abs(fd - ad) / scale
        worst = gap if not np.isfinite(gap) else max(worst, gap)  # a NaN gap must not compare away
        if not np.isfinite(worst):
            break
    return worst


@pytest.mark.parametrize("name", ["euler2d_rk2", "heat3d_fe", "periodic_vortex_rk2", "refined_rk2", "euler2d_llf_rk2",
                                  "refined_llf_rk2"])
def test_adjoint_matches_finite_differences(name):
    """32 random directions, central differences of the GPU frozen-dt map."""
    assert fd_worst(name, 1e-6) <= 1e-6


@pytest.mark.parametrize("name", ["euler2d_fe", "euler3d_rk2", "heat3d_rk2"])
def test_checkpoint_interval_does_not_change_gradient(name):
    _, g, q1, lam = setup(name)
    grads = []
    for every in (1, 4, NSTEPS):
        g.set_state(q1, 0)
        g.reset_time()
        grads.append(g.adjoint(NSTEPS, lam, every=every)[0])
    for gr in grads[1:]:
        assert np.array_equal(gr, grads[0])


@pytest.mark.parametrize("name", ["euler2d_rk2", "euler2d_fe"])
def test_adjoint_leaves_solver_at_step_n(name):
    """h3c_adjoint's forward is the solver's own step: the state, time and
    step afterwards equal those of h3c_solve."""
    o, g, q1, lam = setup(name)
    g.adjoint(NSTEPS, lam, every=3)
    _, g2, _, _ = setup(name)
    g2.solve(NSTEPS)
    fg = o.first_ghost
    assert np.abs(g.state(0)[:, :fg] - g2.state(0)[:, :fg]).max() <= 1e-13 * np.abs(g2.state(0)).max()
    assert g.step() == g2.step() == NSTEPS
    assert abs(g.time() - g2.time()) <= 1e-15 * g2.time()
    g.solve(2)
    g2.solve(2)
    assert abs(g.dt() - g2.dt()) <= 1e-13 * g2.dt()


def test_device_cotangent_and_automatic_interval():
    """CUDA-tensor cotangent/gradient (device pointers through the ABI) and
    the library-chosen checkpoint interval give the host-array result."""
    import torch
    _, g, q1, lam = setup("euler3d_rk2")
    ref, dts_ref = g.adjoint(NSTEPS, lam, every=3)
    g.set_state(q1, 0)
    g.reset_time()
    grad, dts = g.adjoint(NSTEPS, torch.from_numpy(lam).cuda(), every=0)
    assert grad.is_cuda
    assert np.array_equal(grad.cpu().numpy(), ref)
    assert np.array_equal(dts, dts_ref)


def test_solve_dt_matches_oracle_forced_steps():
    o, g, q1, _ = setup("euler3d_rk2")
    dts = [2e-3, 1.5e-3, 2.5e-3, 1e-3]
    g.solve_dt(dts)
    for d in dts:
        o.force_dt(d)
        o.solve(1)
    fg = o.first_ghost
    a, b = g.state(0)[:, :fg], o.state(0)[:, :fg]
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_autograd_function():
    import torch
    from hom3_b200.autograd import solve
    o, g, q1, lam = setup("euler2d_rk2")
    fg = o.first_ghost
    q0 = torch.tensor(q1, requires_grad=True)
    qn = solve(q0, g, NSTEPS, every=4)
    loss = (qn * torch.from_numpy(lam)).sum()
    loss.backward()
    _, g2, _, _ = setup("euler2d_rk2")
    grad, _ = g2.adjoint(NSTEPS, lam, every=4)
    assert np.array_equal(q0.grad.numpy(), grad)
    _, g3, _, _ = setup("euler2d_rk2")
    g3.solve(NSTEPS)
    assert np.abs(qn.detach().numpy()[:, :fg] - g3.state(0)[:, :fg]).max() <= 1e-13 * np.abs(q1).max()


@pytest.mark.parametrize("name", ["euler2d_fe", "euler2d_rk2", "euler3d_rk2", "euler_dirichlet_rk2",
                                  "periodic_vortex_rk2", "refined_fe", "refined_rk2"])
def test_tile_adjoint_matches_per_cell_gather(name):
    """The Euler adjoint stage on Morton tiles (in-tile faces reversed once,
    halves handed over through shared memory) against the per-cell gather
    that reverses every face from both sides: the same sums in another
    order (the forward's stage kernel follows the option as well)."""
    from hom3_b200 import _ffi as F
    o, g, q1, lam = setup(name)
    fg = o.first_ghost
    out = {}
    for tile in (1, 0):
        g.set_option(F.OPT_TILE_KERNEL, tile)
        g.set_state(q1, 0)
        g.reset_time()
        out[tile] = g.adjoint(NSTEPS, lam, every=4)
    # the option switches the forward's stage kernel too (same sums, other order)
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-13 * out[0][1].max()
    scale = np.abs(out[0][0][:, :fg]).max()
    assert np.abs(out[1][0][:, :fg] - out[0][0][:, :fg]).max() <= 1e-12 * scale


def test_tile_adjoint_on_a_large_refined_tree():
    """Many tiles, tile-border, ghost and coarse/fine faces (3D, +2 levels):
    tile kernel against the per-cell gather after 6 RK2 steps."""
    from hom3_b200 import _ffi as F
    _, (o,) = cases.refined_case(level=4, fine=6)
    q1 = cases.smooth_state(o)
    o.set_state(q1)
    g = cases.gpu_solver_from_oracle(o)
    fg = o.first_ghost
    lam = np.zeros_like(q1)
    lam[:, :fg] = np.random.default_rng(3).standard_normal((q1.shape[0], fg))
    out = {}
    for tile in (1, 0):
        g.set_option(F.OPT_TILE_KERNEL, tile)
        g.set_state(q1, 0)
        g.reset_time()
        out[tile] = g.adjoint(6, lam, every=0)[0]
    scale = np.abs(out[0][:, :fg]).max()
    assert np.abs(out[1][:, :fg] - out[0][:, :fg]).max() <= 1e-12 * scale


def test_unsupported_configurations_are_rejected():
    import hom3_b200 as hb
    _, (o,) = cases.advection_case(level=4)
    g = cases.gpu_solver_from_oracle(o)
    with pytest.raises(hb.H3cError):
        g.adjoint(2, np.zeros((o.nv, o.ncells)))


@pytest.mark.parametrize("name", ["euler2d_rk3", "heat3d_rk3", "periodic_vortex_rk3"])
def test_ssprk3_adjoint_matches_dual_oracle(name):
    """EXTENSION: the adjoint of the three SSP-RK3 stages."""
    BUILDERS.update({
        "euler2d_rk3": lambda: cases.euler_case("sod", nd=2, level=5, ti=h3o.SSPRK3),
        "heat3d_rk3": lambda: cases.heat_case(level=3, ti=h3o.SSPRK3),
        "periodic_vortex_rk3": lambda: cases.periodic_vortex_case(level=5, ti=h3o.SSPRK3),
    })
    test_adjoint_matches_dual_oracle(name)


MUSCL_BUILDERS = {
    "vortex_muscl_rk2": lambda: cases.periodic_vortex_case(level=5, recon=h3o.RECON_MUSCL),
    "vortex_muscl_rk3": lambda: cases.periodic_vortex_case(level=5, ti=h3o.SSPRK3, recon=h3o.RECON_MUSCL),
    "sod2d_muscl_fe": lambda: cases.euler_case("sod", nd=2, level=5, ti=h3o.EULER_FORWARD, recon=h3o.RECON_MUSCL),
    "dirichlet_muscl_rk2": lambda: cases.euler_dirichlet_case(nd=2, level=4, ti=h3o.RK2, recon=h3o.RECON_MUSCL),
    "refined_muscl_rk2": lambda: cases.refined_case(ti=h3o.RK2, recon=h3o.RECON_MUSCL),
}


@pytest.mark.parametrize("name", sorted(MUSCL_BUILDERS))
def test_muscl_adjoint_matches_dual_oracle(name):
    """EXTENSION: the adjoint of the MUSCL stage (LSQ gradients, Venkatakrishnan
    limiter differentiated where smooth, its switches frozen) against the
    dual-number oracle, which differentiates the same branches."""
    BUILDERS.update(MUSCL_BUILDERS)
    test_adjoint_matches_dual_oracle(name)


@pytest.mark.parametrize("name", ["vortex_muscl_rk2", "vortex_muscl_rk3"])
def test_muscl_adjoint_matches_finite_differences(name):
    """32 random directions; the step is smaller than the distance of the state
    to the nearest limiter switch (beyond it the map has kinks)."""
    BUILDERS.update(MUSCL_BUILDERS)
    assert fd_worst(name, 1e-7) <= 1e-6


CNS_BUILDERS = {
    "cns_walls_fe": lambda: cases.cns_case("walls", level=4),
    "cns_slip_rk2": lambda: cases.cns_case("slip", level=4, ti=h3o.RK2),
    "cns_isothermal_fe": lambda: cases.cns_case("isothermal", level=4),
    "tgv_cns_rk2": lambda: cases.tgv_case(level=3),
}


@pytest.mark.parametrize("name", sorted(CNS_BUILDERS))
def test_cns_adjoint_matches_dual_oracle(name):
    """The adjoint of the CNS stage (AUSM + three-point viscous flux, cell
    slopes, inflow / outflow / wall conditions, periodic) against the
    dual-number oracle."""
    BUILDERS.update(CNS_BUILDERS)
    test_adjoint_matches_dual_oracle(name)


@pytest.mark.parametrize("name", ["cns_walls_fe", "tgv_cns_rk2"])
def test_cns_adjoint_matches_finite_differences(name):
    BUILDERS.update(CNS_BUILDERS)
    assert fd_worst(name, 1e-6) <= 1e-6


# ---- adjoint of the coupled conjugate-heat loop ----
def cht_setup(level=6, kappa=10.0):
    _, (cns, heat) = cases.cht_case(level=level, kappa=kappa, heat_T=1.3)
    qf, qs = cases.smooth_state(cns), cases.smooth_state(heat)
    cns.set_state(qf)
    heat.set_state(qs)
    gc, gh = cases.gpu_solver_from_oracle(cns), cases.gpu_solver_from_oracle(heat)
    gc.set_partner(gh, cns.partner_cells())
    gh.set_partner(gc, heat.partner_cells())
    return cns, heat, gc, gh, qf, qs


def cht_J(gc, gh, qf, qs, dts, lf, ls):
    gc.set_state(qf, 0)
    gh.set_state(qs, 0)
    gc.reset_time()
    gh.reset_time()
    for i in range(dts.shape[1]):
        gc.solve_dt([dts[0, i]])
        gh.solve_dt([dts[1, i]])
    return float((gc.state(0) * lf).sum() + (gh.state(0) * ls).sum())


@pytest.mark.parametrize("kappa", [0.0, 10.0])
def test_cht_adjoint_matches_finite_differences(kappa):
    """The coupled loop (fluid wall reads the solid, solid ghost reads the
    fluid after its step): fluid and solid directions together, and solid-only
    directions (the gradient with respect to the solid's initial temperature)."""
    import hom3_b200 as hb
    cns, heat, gc, gh, qf, qs = cht_setup(kappa=kappa)
    fgf, fgs = cns.first_ghost, heat.first_ghost
    rng = np.random.default_rng(3)
    lf = np.zeros_like(qf)
    ls = np.zeros_like(qs)
    lf[:, :fgf] = rng.standard_normal((qf.shape[0], fgf))
    ls[:, :fgs] = rng.standard_normal((1, fgs))
    n = 8
    gf, gs, dts = hb.cht_adjoint(0.01, gc, gh, n, lf, ls, every=3)
    assert np.isfinite(gf).all() and np.isfinite(gs).all()
    worst = 0.0
    for k in range(16):
        df = np.zeros_like(qf)
        ds = np.zeros_like(qs)
        if k % 2 == 0:
            df[:, :fgf] = rng.standard_normal((qf.shape[0], fgf))
        ds[:, :fgs] = rng.standard_normal((1, fgs))
        eps = 1e-6
        fd = (cht_J(gc, gh, qf + eps * df, qs + eps * ds, dts, lf, ls)
              - cht_J(gc, gh, qf - eps * df, qs - eps * ds, dts, lf, ls)) / (2 * eps)
        ad = (gf * df).sum() + (gs * ds).sum()
        scale = np.abs(gf * df).sum() + np.abs(gs * ds).sum()
        worst = max(worst, abs(fd - ad) / scale)
    assert worst <= 1e-6, worst


def test_cht_adjoint_forward_is_the_coupled_loop():
    import hom3_b200 as hb
    cns, heat, gc, gh, qf, qs = cht_setup()
    _, _, gc2, gh2, _, _ = cht_setup()
    lf = np.zeros_like(qf)
    ls = np.zeros_like(qs)
    hb.cht_adjoint(0.01, gc, gh, 5, lf, ls, every=2)
    for _ in range(5):
        hb.couple_cht(0.01, gc2, gh2)
        gc2.solve(1)
        gh2.solve(1)
    assert np.array_equal(gc.state(0)[:, :cns.first_ghost], gc2.state(0)[:, :cns.first_ghost])
    assert np.array_equal(gh.state(0)[:, :heat.first_ghost], gh2.state(0)[:, :heat.first_ghost])
    assert gc.step() == 5 and gh.step() == 5


@pytest.mark.parametrize("name", sorted(CNS_BUILDERS))
def test_cns_adjoint_reverse_equals_dual_evaluation(name):
    """The hand-written reverse of the CNS face flux (AUSM + viscous, one
    forward and one reverse sweep per face) against the forward-mode dual
    evaluation of the same flux it replaced: the same derivatives to rounding."""
    from hom3_b200 import _ffi as F
    BUILDERS.update(CNS_BUILDERS)
    o, g, q1, lam = setup(name)
    fg = o.first_ghost
    grad_rev, dts = g.adjoint(NSTEPS, lam, every=5)
    g.set_state(q1, 0)
    g.reset_time()
    g.set_option(F.OPT_CNS_ADJOINT_DUAL, 1)
    grad_dual, dts2 = g.adjoint(NSTEPS, lam, every=5)
    assert np.array_equal(dts, dts2)
    scale = np.abs(grad_dual[:, :fg]).max()
    assert np.max(np.abs(grad_rev[:, :fg] - grad_dual[:, :fg])) <= 1e-12 * scale


def test_cht_adjoint_reverse_equals_dual_evaluation():
    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    cns, heat, gc, gh, qf, qs = cht_setup()
    rng = np.random.default_rng(7)
    lf = np.zeros_like(qf)
    ls = np.zeros_like(qs)
    lf[:, :cns.first_ghost] = rng.standard_normal((qf.shape[0], cns.first_ghost))
    ls[:, :heat.first_ghost] = rng.standard_normal((1, heat.first_ghost))
    gf1, gs1, dts1 = hb.cht_adjoint(0.01, gc, gh, 6, lf, ls, every=4)
    _, _, gc2, gh2, _, _ = cht_setup()
    gc2.set_option(F.OPT_CNS_ADJOINT_DUAL, 1)
    gf2, gs2, dts2 = hb.cht_adjoint(0.01, gc2, gh2, 6, lf, ls, every=4)
    assert np.array_equal(dts1, dts2)
    assert np.max(np.abs(gf1 - gf2)) <= 1e-12 * np.abs(gf2).max()
    assert np.max(np.abs(gs1 - gs2)) <= 1e-12 * np.abs(gs2).max()


def test_autograd_function_cuda_tensors_stay_on_device():
    """With CUDA tensors the state, output, cotangent and gradient move device
    to device; the results are the host path's."""
    import torch
    from hom3_b200.autograd import solve
    o, g, q1, lam = setup("euler2d_rk2")
    q0 = torch.tensor(q1, device="cuda", requires_grad=True)
    qn = solve(q0, g, NSTEPS, every=4)
    assert qn.is_cuda
    loss = (qn * torch.from_numpy(lam).cuda()).sum()
    loss.backward()
    assert q0.grad.is_cuda
    _, g2, _, _ = setup("euler2d_rk2")
    grad, _ = g2.adjoint(NSTEPS, lam, every=4)
    assert np.array_equal(q0.grad.cpu().numpy(), grad)
    _, g3, _, _ = setup("euler2d_rk2")
    g3.solve(NSTEPS)
    assert np.array_equal(qn.detach().cpu().numpy(), g3.state(0))


def test_state_round_trip_through_device_memory():
    import torch
    o, g, q1, _ = setup("euler2d_rk2")
    t = torch.tensor(q1, device="cuda")
    g.set_state(t, 0)
    back = torch.empty_like(t)
    g.state(0, out=back)
    assert torch.equal(back, t)
    assert np.array_equal(g.state(0), q1)
