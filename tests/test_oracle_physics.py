"""Known-answer checks of the oracle's finite-volume arithmetic (hom3's own
solver tests carry no numeric assertions, so these pin the restatement)."""
import math

import numpy as np
import pytest

import cases
from oracle import h3o


def test_constant_state_preserved_exactly():
    """euler_fv_solver_test.cpp:82-84: the solution is the initial condition for all t."""
    _, (o,) = cases.euler_case("constant", nd=3, level=3)
    q0 = o.state(0)[:, : o.first_ghost].copy()
    o.solve(20)
    assert np.array_equal(o.state(0)[:, : o.first_ghost], q0)


def test_cns_free_stream_preserved():
    """cns_fv_solver_test.cpp:91-141: free-stream state with Neumann conditions."""
    _, (o,) = cases.cns_case("constant", level=4)
    q0 = o.state(0)[:, : o.first_ghost].copy()
    o.solve(10)
    assert np.max(np.abs(o.state(0)[:, : o.first_ghost] - q0)) <= 1e-14


@pytest.mark.parametrize("case", ["tgv", "periodic_vortex"])
def test_periodic_conservation(case):
    """A periodic domain exchanges no flux with the outside: the sums of the
    conserved variables stay constant to rounding."""
    _, (o,) = cases.tgv_case(level=3) if case == "tgv" else cases.periodic_vortex_case(level=5)
    fg = o.first_ghost
    vol = o.tables()["length"][:fg] ** o.w.nd
    s0 = (o.state(0)[:, :fg] * vol).sum(1)
    o.solve(6)
    s1 = (o.state(0)[:, :fg] * vol).sum(1)
    scale = np.abs(o.state(0)[:, :fg] * vol).sum(1)
    assert np.all(np.abs(s1 - s0) <= 1e-13 * scale)


def test_refined_tree_conserves():
    """EXTENSION: coarse/fine faces are conservative (both sides use one flux):
    while the cells next to the outer faces are still untouched (no flux
    through the domain boundary), the conserved sums do not change."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 5)
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
    o = w.add_solver(h3o.EULER, h3o.AUSM, h3o.EULER_FORWARD, bcs=bcs, ic_kind=h3o.IC_EXPLOSION,
                     ic=[0.5, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1], time_end=1.0, cfl=0.4)
    o.initialize()
    fg = o.first_ghost
    t = o.tables()
    vol = t["length"][:fg] ** 3
    outer = (t["neighbors"][:, :fg] >= fg).any(0) & (t["neighbors"][:, :fg] < t["ncells"]).any(0)
    q0 = o.state(0)[:, :fg].copy()
    s0 = (q0 * vol).sum(1)
    checked = 0
    for _ in range(6):
        o.solve(1)
        q = o.state(0)[:, :fg]
        if not np.array_equal(q[:, outer], q0[:, outer]):
            break
        s1 = (q * vol).sum(1)
        scale = np.abs(q * vol).sum(1)
        assert np.all(np.abs(s1 - s0) <= 1e-14 * scale)
        checked += 1
    assert checked >= 2


def _exact_sod(x, t, x0=0.3, L=(1.0, 0.75, 1.0), R=(0.125, 0.0, 0.1), g=1.4):
    """Exact Riemann solution (Toro, Riemann Solvers and Numerical Methods for
    Fluid Dynamics, ch. 4: pressure function and Newton iteration for p*)."""
    rl, ul, pl = L
    rr, ur, pr = R
    al, ar = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)

    def f(p, rk, pk, ak):
        if p > pk:
            A, B = 2 / ((g + 1) * rk), (g - 1) / (g + 1) * pk
            return (p - pk) * math.sqrt(A / (p + B)), math.sqrt(A / (B + p)) * (1 - (p - pk) / (2 * (B + p)))
        r = p / pk
        return 2 * ak / (g - 1) * (r ** ((g - 1) / (2 * g)) - 1), 1 / (rk * ak) * r ** (-(g + 1) / (2 * g))

    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = f(p, rl, pl, al)
        fr, dr = f(p, rr, pr, ar)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(1e-8, p - dp)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = f(p, rl, pl, al)
    fr, _ = f(p, rr, pr, ar)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    out = np.empty_like(x)
    for i, xi in enumerate(x):
        s = (xi - x0) / t
        if s < u:  # left of contact
            if p > pl:
                sl = ul - al * math.sqrt((g + 1) / (2 * g) * p / pl + (g - 1) / (2 * g))
                out[i] = rl if s < sl else rl * ((p / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pl + 1))
            else:
                shl, stl = ul - al, u - al * (p / pl) ** ((g - 1) / (2 * g))
                if s < shl:
                    out[i] = rl
                elif s > stl:
                    out[i] = rl * (p / pl) ** (1 / g)
                else:
                    out[i] = rl * (2 / (g + 1) + (g - 1) / ((g + 1) * al) * (ul - s)) ** (2 / (g - 1))
        else:
            if p > pr:
                sr = ur + ar * math.sqrt((g + 1) / (2 * g) * p / pr + (g - 1) / (2 * g))
                out[i] = rr if s > sr else rr * ((p / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pr + 1))
            else:
                shr, str_ = ur + ar, u + ar * (p / pr) ** ((g - 1) / (2 * g))
                if s > shr:
                    out[i] = rr
                elif s < str_:
                    out[i] = rr * (p / pr) ** (1 / g)
                else:
                    out[i] = rr * (2 / (g + 1) - (g - 1) / ((g + 1) * ar) * (ur - s)) ** (2 / (g - 1))
    return out


def test_sod_converges_to_exact_riemann_solution():
    """euler_fv_solver_test.cpp:114-156 cite Toro's modified Sod problem; the
    first-order AUSM solution's L1 density error against the exact solution
    must fall with refinement (first-order rate)."""
    errs = []
    for level in (5, 6, 7):
        w = h3o.World(2, [0, 0], [1, 1], level=level)
        bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
        o = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_SHOCK_TUBE, ic=cases.SOD,
                         time_end=0.2, cfl=0.4)
        o.initialize()
        while o.time() < 0.2:
            o.solve(1)
        fg = o.first_ghost
        t = o.tables()
        x = t["x_center"][0, :fg]
        rho = o.state(0)[2, :fg]
        errs.append(np.mean(np.abs(rho - _exact_sod(x, o.time()))))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 0.02
    assert errs[1] / errs[2] > 1.4


def _vortex_l2_error(level, recon, ti, t_end=2.0):
    """Density L2 error of the periodic isentropic vortex (beta 5, u = v = 1 on
    [0, 10]^2) at t_end against the exact solution (the initial vortex moved by
    (t_end, t_end)), both as cell averages."""
    w = h3o.World(2, [0, 0], [10, 10], level=level)
    bcs = [h3o.bc(h3o.BC_PERIODIC, g) for g in w.cube_boundaries()]
    o = w.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=bcs, ic_kind=h3o.IC_VORTEX_PARAM, ic=[5.0, 5.0, 5.0, 1.0, 1.0],
                     time_end=t_end, recon=recon, **dict(cases.EULER_PROPS, cfl=0.5))
    o.initialize()
    w2 = h3o.World(2, [0, 0], [10, 10], level=level)
    e = w2.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=[h3o.bc(h3o.BC_PERIODIC, g) for g in w2.cube_boundaries()],
                      ic_kind=h3o.IC_VORTEX_PARAM, ic=[5.0, 5.0 + t_end, 5.0 + t_end, 1.0, 1.0], time_end=t_end,
                      **cases.EULER_PROPS)
    e.initialize()
    while o.time() < t_end - 1e-12:
        o.solve(1)
    fg = o.first_ghost
    return float(np.sqrt(((o.state(0)[2, :fg] - e.state(0)[2, :fg]) ** 2).mean()))


def test_muscl_ssprk3_is_second_order_on_the_vortex():
    """EXTENSION (not in hom3): LSQ gradients + MUSCL + Venkatakrishnan with
    SSP-RK3 converge at second order on the smooth vortex (error ratio per
    refinement near 4; the first-order scheme stays below 2)."""
    e2 = [_vortex_l2_error(lv, h3o.RECON_MUSCL, h3o.SSPRK3) for lv in (5, 6)]
    e1 = [_vortex_l2_error(lv, h3o.RECON_NONE, h3o.RK2) for lv in (5, 6)]
    assert e2[0] / e2[1] > 3.3, e2
    assert e1[0] / e1[1] < 2.0, e1
    assert e2[1] < e1[1] / 5


@pytest.mark.parametrize("ti", [h3o.RK2, h3o.SSPRK3])
def test_muscl_conserves_on_refined_periodic_tree(ti):
    """EXTENSION: MUSCL on a periodic 2:1 tree with coarse/fine faces keeps the
    conserved sums to rounding (one face point and one F(l, r) per face)."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=3)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, 5)
    bcs = [h3o.bc(h3o.BC_PERIODIC, g) for g in w.cube_boundaries()]
    o = w.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=bcs, ic_kind=h3o.IC_EXPLOSION,
                     ic=[0.5, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1], time_end=1.0, cfl=0.4, recon=h3o.RECON_MUSCL)
    o.initialize()
    fg = o.first_ghost
    vol = o.tables()["length"][:fg] ** 3
    s0 = (o.state(0)[:, :fg] * vol).sum(1)
    o.solve(6)
    q = o.state(0)[:, :fg]
    s1 = (q * vol).sum(1)
    scale = np.abs(q * vol).sum(1)
    assert np.all(np.abs(s1 - s0) <= 1e-13 * scale)


def test_muscl_preserves_constant_state():
    _, (o,) = cases.euler_case("constant", nd=3, level=3, ti=h3o.SSPRK3, recon=h3o.RECON_MUSCL)
    q0 = o.state(0)[:, : o.first_ghost].copy()
    o.solve(5)
    assert np.max(np.abs(o.state(0)[:, : o.first_ghost] - q0)) <= 1e-14


def test_conductivity_ratio_weights_interface_temperature():
    """EXTENSION: with kappa = k_solid / k_fluid the interface temperature is
    (T_f + kappa T_s) / (1 + kappa): a very conductive solid pins the fluid
    wall temperature near its own, so the fluid near the solid heats faster
    than with hom3's mean (kappa = 1)."""
    res = {}
    for kappa in (1.0, 50.0):
        _, (cns, heat) = cases.cht_case(level=6, kappa=kappa, heat_T=1.3)
        for _ in range(5):
            h3o.couple_cht(cns, heat, 0.01)
            cns.solve()
            heat.solve()
        q = cns.state(0)[:, : cns.first_ghost]
        T = 1.4 * 0.4 * (q[3] - 0.5 * (q[0] ** 2 + q[1] ** 2) / q[2]) / q[2]
        res[kappa] = T.max()
    assert res[50.0] > res[1.0]


# ---- advection (advection/physics.hpp, advection/boundary_conditions.hpp) ----
def _lattice(o):
    """(i, j) lattice index of every interior cell of a uniform 2D grid."""
    t = o.tables()
    fg = o.first_ghost
    h = t["length"][0]
    ij = np.floor(t["x_center"][:, :fg] / h).astype(int)
    return ij, int(round(1 / h))


def test_advection_upwind_at_cfl_one_shifts_by_one_cell():
    """u = (1, 0), CFL 1: dt = h, and the upwind update q - (q - q_left) moves
    the state exactly one cell per step (to rounding), periodic in x."""
    _, (o,) = cases.advection_case(level=5, bc_kind=h3o.BC_PERIODIC, vel_kind=h3o.VEL_CONSTANT, vel=(1.0, 0.0))
    ij, n = _lattice(o)
    fg = o.first_ghost
    q0 = np.empty((n, n))
    q0[ij[0], ij[1]] = o.state(0)[0, :fg]
    o.solve(7)
    assert abs(o.dt() - 1.0 / n) <= 1e-15
    q = np.empty((n, n))
    q[ij[0], ij[1]] = o.state(0)[0, :fg]
    assert np.abs(q - np.roll(q0, 7, axis=0)).max() <= 1e-15


def test_advection_upwind_reproduces_hom3_sign_for_negative_velocity():
    """hom3's upwind flux is u_L q_L negated when the face velocity is
    negative (advection/physics.hpp:132-145), not u_R q_R: with u = (-1, 0)
    at CFL 1 every face carries +q_L and the state moves one cell in +x."""
    _, (o,) = cases.advection_case(level=5, bc_kind=h3o.BC_PERIODIC, vel_kind=h3o.VEL_CONSTANT, vel=(-1.0, 0.0))
    ij, n = _lattice(o)
    fg = o.first_ghost
    q0 = np.empty((n, n))
    q0[ij[0], ij[1]] = o.state(0)[0, :fg]
    o.solve(1)
    q = np.empty((n, n))
    q[ij[0], ij[1]] = o.state(0)[0, :fg]
    assert np.abs(q - np.roll(q0, 1, axis=0)).max() <= 1e-15


@pytest.mark.parametrize("flux", [h3o.LLF, h3o.UPWIND])
def test_advection_conserves_on_periodic_domain(flux):
    """Both fluxes are face fluxes F(l, r) shared by the two cells: the sum of
    q h^2 is conserved on a periodic domain (rotating field, RK2)."""
    _, (o,) = cases.advection_case(level=5, flux=flux, ti=h3o.RK2, bc_kind=h3o.BC_PERIODIC, cfl=0.4)
    fg = o.first_ghost
    h2 = o.tables()["length"][:fg] ** 2
    m0 = (o.state(0)[0, :fg] * h2).sum()
    o.solve(20)
    assert abs((o.state(0)[0, :fg] * h2).sum() - m0) <= 1e-13 * abs(m0)


def test_advection_llf_is_bounded_for_a_uniform_velocity():
    """LLF with a uniform velocity is the monotone upwind scheme: at CFL 0.4 per
    direction the state stays within the initial bounds."""
    _, (o,) = cases.advection_case(level=5, flux=h3o.LLF, bc_kind=h3o.BC_PERIODIC, vel_kind=h3o.VEL_CONSTANT,
                                   vel=(0.6, -0.8), cfl=0.4)
    fg = o.first_ghost
    o.solve(30)
    q = o.state(0)[0, :fg]
    assert q.min() >= 0.1 - 1e-14 and q.max() <= 1.0 + 1e-14


def test_advection_conditions():
    """Ghost values: Dirichlet 2 v - q_b, Neumann q_b - |x_b - x_g| g, and the
    characteristic condition, whose inflow and outflow branches both give q_b."""
    for kind in (h3o.BC_ADV_DIRICHLET, h3o.BC_ADV_NEUMANN, h3o.BC_ADV_CHARACTERISTIC):
        _, (o,) = cases.advection_case(level=4, bc_kind=kind)
        t = o.tables()
        fg = o.first_ghost
        o.apply_bcs(0)
        q = o.state(0)[0]
        info = o.info()
        for gcell in range(fg, o.ncells):
            b = next(int(n) for n in t["neighbors"][:, gcell] if 0 <= n < o.ncells)
            v = info["bcs"][t["bc_idx"][gcell]][1][0]
            if kind == h3o.BC_ADV_DIRICHLET:
                want = 2 * v - q[b]
            elif kind == h3o.BC_ADV_NEUMANN:
                want = q[b] - np.linalg.norm(t["x_center"][:, b] - t["x_center"][:, gcell]) * v
            else:
                want = q[b]
            assert q[gcell] == want, (kind, gcell)


def test_advection_time_step():
    """compute_dt: CFL h / max_d |u_d(x_c)| (advection/physics.hpp:78-87), min over cells."""
    _, (o,) = cases.advection_case(level=4, cfl=0.7)
    t = o.tables()
    fg = o.first_ghost
    u = o.velocity()[:, :fg]
    want = (0.7 * t["length"][:fg] / np.abs(u).max(axis=0)).min()
    assert abs(o.min_dt() - want) <= 1e-15 * want


def test_advection_bench_inputs_match_the_oracle():
    """The advection workload's velocity field and initial disc (hom3_b200.workloads)
    against the oracle's restatement of hom3's test: velocity to rounding of the
    trigonometric functions, cell averages exactly."""
    import hom3_b200 as hb
    from hom3_b200 import workloads as W
    _, (o,) = cases.advection_case(level=6)
    t = o.tables()
    fg = o.first_ghost
    assert np.abs(W.rotation_velocity(t["x_center"]) - o.velocity()).max() <= 1e-15
    q = hb.cell_average(W.disc_ic(), t["x_center"][:, :fg], t["length"][:fg], 2)
    assert np.array_equal(q[0], o.state(0)[0, :fg])
