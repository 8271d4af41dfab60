"""Test cases mirroring hom3's own solver tests, built in the oracle.

Each builder returns (world, [solvers]) after initialize().  Cases follow
src/solver/fv/euler/tests/euler_fv_solver_test.cpp, cns/tests/cns_fv_solver_test.cpp,
heat/tests/heat_fv_solver_test.cpp, tests/coupled_cns_heat_test.cpp and
euler/tests/coupled_euler_euler_test.cpp, at reduced refinement levels where
noted so the oracle finishes in seconds.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import h3o  # noqa: E402

EULER_PROPS = dict(gamma=1.4, Minfty=0.1, cfl=0.2, Rspecific=287.058, T0=273.15, rho0=1.225)
SOD = [0, 0, 0.3, 1.0, 0.75, 1.0, 0.125, 0.0, 0.1]
P123 = [0, 0, 0.5, 1.0, -2.0, 0.4, 1.0, 2.0, 0.4]


def neumann_cube(w):
    return [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]


def euler_case(name, nd=3, level=4, ti=h3o.EULER_FORWARD, flux=h3o.AUSM, **extra):
    """euler_fv_solver_test.cpp:85-286 (3D cases at level 4 instead of 5).
    extra: EXTENSION keywords (recon, limiter_k)."""
    if name == "vortex":
        w = h3o.World(2, [-8, -8], [8, 8], level=level)
        bcs = [h3o.bc(h3o.BC_EULER_VORTEX, g) for g in w.cube_boundaries()]
        s = w.add_solver(h3o.EULER, flux, ti, bcs=bcs, ic_kind=h3o.IC_VORTEX, time_end=2.0, **EULER_PROPS, **extra)
    else:
        lo, hi = [0.0] * nd, [1.0] * nd
        w = h3o.World(nd, lo, hi, level=level)
        if name == "constant":
            ic_kind, ic, tend = h3o.IC_CONSTANT_PV, [0.5] * nd + [1.0, 1.0], 0.25
        elif name == "sod":
            ic_kind, ic, tend = h3o.IC_SHOCK_TUBE, SOD, 0.2
        elif name == "p123":
            ic_kind, ic, tend = h3o.IC_SHOCK_TUBE, P123, 0.15
        elif name == "explosion":
            ic_kind, ic, tend = h3o.IC_EXPLOSION, [0.5, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1], 0.25
        else:
            raise KeyError(name)
        s = w.add_solver(h3o.EULER, flux, ti, bcs=neumann_cube(w), ic_kind=ic_kind, ic=ic, time_end=tend,
                         **EULER_PROPS, **extra)
    s.initialize()
    return w, [s]


def euler_dirichlet_case(nd=2, level=5, ti=h3o.EULER_FORWARD, **extra):
    """Dirichlet / non-zero Neumann conditions (euler/boundary_conditions.hpp:17-67)."""
    w = h3o.World(nd, [0.0] * nd, [1.0] * nd, level=level)
    g = w.cube_boundaries()
    state = [0.1, 0.0, 1.0, 2.5] if nd == 2 else [0.1, 0.0, 0.0, 1.0, 2.5]
    flux = [0.01 * (i + 1) for i in range(nd + 2)]
    bcs = [h3o.bc(h3o.BC_EULER_DIRICHLET, g[0], state), h3o.bc(h3o.BC_EULER_NEUMANN, g[1], flux)]
    bcs += [h3o.bc(h3o.BC_EULER_NEUMANN, x) for x in g[2:]]
    s = w.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=bcs, ic_kind=h3o.IC_SHOCK_TUBE, ic=SOD, time_end=0.2,
                     **EULER_PROPS, **extra)
    s.initialize()
    return w, [s]


CNS_PROPS = dict(gamma=1.4, cfl=0.4, cfl_viscous=0.4, Rspecific=287.058, T0=273.15, rho0=1.225, Pr0=0.72,
                 Sutherland0=110.4)


def cns_case(name, level=6, ti=h3o.EULER_FORWARD):
    """cns_fv_solver_test.cpp:91-211 (constant_ic, sod_shock_tube_ic; level 6 instead of 8)."""
    if name in ("constant", "sod"):
        w = h3o.World(2, [0, 0], [1, 1], level=level)
        probe = w.add_solver(h3o.CNS, h3o.AUSM, ti, bcs=neumann_cube(w), ic_kind=h3o.IC_CONSTANT_PV,
                             ic=[0, 0, 1, 1], Minfty=0.1, ReInfty=100.0, time_end=0.25, **CNS_PROPS)
        q = probe.quantities()
        w = h3o.World(2, [0, 0], [1, 1], level=level)
        if name == "constant":
            s = w.add_solver(h3o.CNS, h3o.AUSM, ti, bcs=neumann_cube(w), ic_kind=h3o.IC_CONSTANT_PV,
                             ic=[q["u_inf"], 0.0, q["rho_inf"], q["p_inf"]], Minfty=0.1, ReInfty=100.0,
                             time_end=0.25, **CNS_PROPS)
        else:
            ic = [0, 0, 0.3, 1.0 * q["rho_inf"], 0.75 * q["u_inf"], 1.0 * q["p_inf"], 0.125 * q["rho_inf"],
                  0.0, 0.1 * q["p_inf"]]
            s = w.add_solver(h3o.CNS, h3o.AUSM, ti, bcs=neumann_cube(w), ic_kind=h3o.IC_SHOCK_TUBE, ic=ic,
                             Minfty=0.1, ReInfty=1000.0, time_end=0.25, **CNS_PROPS)
        s.initialize()
        return w, [s]
    if name in ("walls", "slip", "isothermal"):
        # inflow / outflow + Neumann far field (cns_fv_solver_test.cpp:212-286, flow_past_cube, with the
        # cube replaced by conditions on the cube faces so a small grid has all kinds)
        w0 = h3o.World(2, [0, 0], [1, 1], level=level)
        probe = w0.add_solver(h3o.CNS, h3o.AUSM, ti, bcs=neumann_cube(w0), ic_kind=h3o.IC_CONSTANT_PV,
                              ic=[0, 0, 1, 1], Minfty=0.2, ReInfty=200.0, **CNS_PROPS)
        q = probe.quantities()
        fs = [q["u_inf"], 0.0, q["rho_inf"], q["p_inf"]]
        w = h3o.World(2, [0, 0], [1, 1], level=level)
        g = w.cube_boundaries()
        wall = {"walls": (h3o.BC_CNS_ADIABATIC_NOSLIP, []), "slip": (h3o.BC_CNS_ADIABATIC_SLIP, []),
                "isothermal": (h3o.BC_CNS_ISOTHERMAL_NOSLIP, [1.05 * q["T_inf"]])}[name]
        bcs = [h3o.bc(h3o.BC_CNS_INFLOW, g[0], fs), h3o.bc(h3o.BC_CNS_OUTFLOW, g[1], fs),
               h3o.bc(wall[0], g[2], wall[1]), h3o.bc(h3o.BC_EULER_NEUMANN, g[3])]
        ic = [0, 0, 0.5, 1.0 * q["rho_inf"], q["u_inf"], q["p_inf"], 0.9 * q["rho_inf"], q["u_inf"], q["p_inf"]]
        s = w.add_solver(h3o.CNS, h3o.AUSM, ti, bcs=bcs, ic_kind=h3o.IC_SHOCK_TUBE, ic=ic, Minfty=0.2,
                         ReInfty=200.0, time_end=100.0, **CNS_PROPS)
        s.initialize()
        return w, [s]
    raise KeyError(name)


def heat_case(level=3, ti=h3o.EULER_FORWARD):
    """heat_fv_solver_test.cpp:81-105 (level 3 instead of 4)."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=level)
    g = w.cube_boundaries()
    bcs = [h3o.bc(h3o.BC_HEAT_DIRICHLET, g[0], [1.0]), h3o.bc(h3o.BC_HEAT_DIRICHLET, g[1], [1.0])]
    bcs += [h3o.bc(h3o.BC_HEAT_NEUMANN, x, [0.0]) for x in g[2:]]
    s = w.add_solver(h3o.HEAT, 0, ti, bcs=bcs, ic_kind=h3o.IC_CONSTANT_CV, ic=[0.0], cfl=0.5, time_end=0.25)
    s.initialize()
    return w, [s]


def cht_case(level=8, kappa=0.0, heat_T=None):
    """coupled_cns_heat_test.cpp:56-248: CNS (solver 0) around a heat-conducting cube (solver 1).
    EXTENSION: kappa = k_solid / k_fluid (0: hom3's mean interface temperature) and a
    solid initial temperature heat_T (default the free-stream T, as in hom3)."""
    lo, hi = [-7.0, -7.0], [7.0, 7.0]
    w = h3o.World(2, lo, hi, level=level, max_solvers=2)
    h = w.cell_length_at_level(level)
    c0, c1, c2 = h3o.make_cube(2, [-3.0, 0.0], [1.0, 1.0], h)
    probe_w = h3o.World(2, lo, hi, level=1)
    probe = probe_w.add_solver(h3o.CNS, h3o.AUSM, h3o.EULER_FORWARD, bcs=neumann_cube(probe_w),
                               Minfty=0.2, ReInfty=100.0, **CNS_PROPS)
    q = probe.quantities()
    fs = [q["u_inf"], 0.0, q["rho_inf"], q["p_inf"]]
    g = w.cube_boundaries()
    cns_bcs = [h3o.bc(h3o.BC_CNS_INFLOW, g[0], fs), h3o.bc(h3o.BC_CNS_OUTFLOW, g[1], fs),
               h3o.bc(h3o.BC_EULER_NEUMANN, g[2]), h3o.bc(h3o.BC_EULER_NEUMANN, g[3]),
               h3o.bc(h3o.BC_CPL_CNS_HEAT, c1, [kappa], partner=1)]
    cns = w.add_solver(h3o.CNS, h3o.AUSM, h3o.EULER_FORWARD, bcs=cns_bcs, domain=c0, domain_kind=1,
                       ic_kind=h3o.IC_CONSTANT_PV, ic=fs, Minfty=0.2, ReInfty=100.0, time_end=10.0,
                       **dict(CNS_PROPS, cfl=0.4))
    heat = w.add_solver(h3o.HEAT, 0, h3o.EULER_FORWARD, bcs=[h3o.bc(h3o.BC_CPL_HEAT_CNS, c2, [kappa], partner=0)],
                        domain=c0, domain_kind=2, ic_kind=h3o.IC_CONSTANT_CV,
                        ic=[q["T_inf"] if heat_T is None else heat_T], cfl=0.5,
                        time_end=10.0)
    heat.initialize()  # initialize(hgrid, heatSolver, cnsSolver): coupled_cns_heat_test.cpp:231
    cns.initialize()
    return w, [cns, heat]


def euler_euler_case(level=4):
    """coupled_euler_euler_test.cpp:94-163 (level 4 instead of 5)."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=level, max_solvers=2)
    h = w.cell_length_at_level(level)
    c0, c1, c2 = h3o.make_cube(3, [0.5, 0.5, 0.5], [0.2, 0.2, 0.2], h, tol=0.5)
    props = dict(EULER_PROPS, Minfty=0.2)
    s0 = w.add_solver(h3o.EULER, h3o.AUSM, h3o.EULER_FORWARD,
                      bcs=neumann_cube(w) + [h3o.bc(h3o.BC_CPL_EULER_EULER, c1, partner=1)],
                      domain=c0, domain_kind=1, ic_kind=h3o.IC_SHOCK_TUBE, ic=SOD, time_end=0.25, **props)
    s1 = w.add_solver(h3o.EULER, h3o.AUSM, h3o.EULER_FORWARD,
                      bcs=[h3o.bc(h3o.BC_CPL_EULER_EULER, c2, partner=0)],
                      domain=c0, domain_kind=2, ic_kind=h3o.IC_SHOCK_TUBE, ic=SOD, time_end=0.25, **props)
    s0.initialize()
    s1.initialize()
    return w, [s0, s1]


# ---------------------------------------------------------------------------
def advection_case(level=7, flux=h3o.UPWIND, ti=h3o.EULER_FORWARD, bc_kind=None, vel_kind=h3o.VEL_ROTATION,
                   vel=(0.5, 0.5, 0.5), nd=2, cfl=1.0, fine=None):
    """advection_fv_solver_test.cpp:51-125: the disc q = 1 (r = 0.08 around (0.25, 0.5)) in q = 0.1,
    carried by the test's rotating velocity field, characteristic conditions on all faces, upwind flux,
    forward Euler, CFL 1 (level 7, as in hom3).  bc_kind / vel_kind select other conditions and fields;
    fine: EXTENSION, refine the r = 0.3 sphere around the centre to that level."""
    w = h3o.World(nd, [0.0] * nd, [1.0] * nd, level=level)
    if fine is not None:
        w.refine_sphere([0.5] * nd, 0.3, fine)
    g = w.cube_boundaries()
    if bc_kind is None or bc_kind == h3o.BC_ADV_CHARACTERISTIC:
        bcs = [h3o.bc(h3o.BC_ADV_CHARACTERISTIC, x) for x in g]
    elif bc_kind == h3o.BC_PERIODIC:
        bcs = [h3o.bc(h3o.BC_PERIODIC, x) for x in g]
    elif bc_kind == h3o.BC_ADV_DIRICHLET:
        bcs = [h3o.bc(h3o.BC_ADV_DIRICHLET, x, [0.1 + 0.05 * i]) for i, x in enumerate(g)]
    else:
        bcs = [h3o.bc(h3o.BC_ADV_NEUMANN, x, [0.02 * (i + 1)]) for i, x in enumerate(g)]
    centre = [0.25, 0.5, 0.5][:nd] + [0.0] * (3 - nd)
    s = w.add_solver(h3o.ADVECTION, flux, ti, bcs=bcs, ic_kind=h3o.IC_DISC, ic=centre + [0.08, 1.0, 0.1],
                     cfl=cfl, time_end=100.0, vel_kind=vel_kind, vel=vel)
    s.initialize()
    return w, [s]


def gpu_solver_from_oracle(o: "h3o.Solver", precision=0):
    """Hand the oracle's (hom3-numbered) tables and initial state to the C ABI:
    the drop-in path a hom3 Solver would take after Solver::initialize."""
    import hom3_b200 as hb
    from hom3_b200.solver import Condition

    info = o.info()
    props = {k: info[k] for k in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")}
    s = hb.Solver(info["nd"], info["physics"], info["flux"], info["ti"], precision, reconstruction=info["recon"],
                  limiter_k=info["limiter_k"], **props)
    t = o.tables()
    s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"],
               [Condition(k, v) for k, v in info["bcs"]], t["subface_cells"])
    if any(k == h3o.BC_PERIODIC for k, _ in info["bcs"]):
        s.set_periodic(o.partner_cells())
    if info["physics"] == h3o.ADVECTION:
        s.set_velocity(o.velocity())
    s.set_state(o.state(0), 0)
    s.reset_time()
    return s


def tgv_case(level=4, ti=h3o.RK2):
    """EXTENSION (not in hom3): 3D Taylor-Green vortex, periodic [0, 2pi]^3,
    Re = 1600, Mach 0.1, Pr = 0.71 (the CNS benchmark configuration)."""
    import math
    w = h3o.World(3, [0, 0, 0], [2 * math.pi] * 3, level=level)
    bcs = [h3o.bc(h3o.BC_PERIODIC, g) for g in w.cube_boundaries()]
    s = w.add_solver(h3o.CNS, h3o.AUSM, ti, bcs=bcs, ic_kind=h3o.IC_TAYLOR_GREEN, ic=[0.1, 1.0, 1 / 1.4],
                     Minfty=0.1, ReInfty=1600.0, Pr0=0.71, cfl=0.5, cfl_viscous=0.4, time_end=10.0,
                     **{k: v for k, v in CNS_PROPS.items() if k not in ("cfl", "cfl_viscous", "Pr0")})
    s.initialize()
    return w, [s]


def periodic_vortex_case(level=6, ti=h3o.RK2, flux=h3o.AUSM, **extra):
    """EXTENSION (not in hom3): the 2D isentropic vortex of the first benchmark
    configuration -- [0, 10]^2, centre (5, 5), beta 5, periodic."""
    w = h3o.World(2, [0, 0], [10, 10], level=level)
    bcs = [h3o.bc(h3o.BC_PERIODIC, g) for g in w.cube_boundaries()]
    s = w.add_solver(h3o.EULER, flux, ti, bcs=bcs, ic_kind=h3o.IC_VORTEX_PARAM, ic=[5.0, 5.0, 5.0, 1.0, 1.0],
                     time_end=10.0, **dict(EULER_PROPS, cfl=0.5), **extra)
    s.initialize()
    return w, [s]


def refined_case(ti=h3o.RK2, level=2, fine=4, **extra):
    """EXTENSION (not in hom3): 3D Sod tube on a tree refined +2 levels in a sphere."""
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=level)
    w.refine_sphere([0.5, 0.5, 0.5], 0.3, fine)
    s = w.add_solver(h3o.EULER, h3o.AUSM, ti, bcs=neumann_cube(w), ic_kind=h3o.IC_SHOCK_TUBE,
                     ic=[0, 0, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1], time_end=1.0, cfl=0.4, **extra)
    s.initialize()
    return w, [s]


def smooth_state(o: "h3o.Solver", seed=0):
    """A state on which the discrete map is smooth, for derivative checks: the
    case's state plus a uniform subsonic drift (Euler; no face sits at the
    interface-Mach-number switch m = 0) and a small per-cell perturbation,
    or 1 + a smooth random field (heat).  gamma = 1.4."""
    q = o.state(0).copy()
    fg = o.first_ghost
    nd = o.w.nd
    rng = np.random.default_rng(seed)
    if o.nv == 1:
        x = o.tables()["x_center"]
        k = rng.integers(1, 4, size=(4, nd))
        ph = rng.uniform(0, 2 * np.pi, size=4)
        f = sum(np.sin(2 * np.pi * (k[m] @ x) + ph[m]) for m in range(4))
        q[0] = 1.0 + 0.1 * f
        return q
    drift = np.array([0.3, 0.1, 0.05][:nd])
    rho = q[nd]
    u = q[:nd] / rho
    p = 0.4 * (q[nd + 1] - 0.5 * rho * (u * u).sum(axis=0))
    # a smooth random perturbation of 1e-3 (random phases): no symmetry of the
    # initial condition makes two neighbours tie (a tie is a kink of the
    # limiter's max / min, where central differences and one-sided derivatives
    # differ), and no per-cell extrema are added
    x = o.tables()["x_center"][:, :q.shape[1]]
    span = np.ptp(x[:, :fg], axis=1).max() + 1e-300

    def field():  # random real wave vectors: no reflection or rotation symmetry survives
        k = rng.uniform(0.5, 2.5, size=(3, nd)) * (2 * np.pi / span)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        return sum(np.sin(k[m] @ x + ph[m]) for m in range(3)) / 3

    rho = rho * (1.0 + 1e-3 * field())
    p = p * (1.0 + 1e-3 * field())
    u = u + drift[:, None] + 1e-3 * np.stack([field() for _ in range(nd)])
    q[:nd] = rho * u
    q[nd] = rho
    q[nd + 1] = p / 0.4 + 0.5 * rho * (u * u).sum(axis=0)
    q[:, fg:] = 0.0
    return q
