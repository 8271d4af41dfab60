"""Synthetic workloads of the benchmark configurations (seeded; no datasets).

riemann3d_refined: 3D Euler on a hierarchical Cartesian tree -- base level 6
(64^3) on the unit cube, refined +2 levels (to level 8) in the sphere of
radius 0.25 at the centre, 2:1 face balanced.  Initial state: Riemann problem
split at x = 0.5 (left rho = 1, p = 1; right rho = 0.125, p = 0.1; u = 0) as
in hom3's shock_tube (euler/initial_conditions.hpp:51-90), with 1%
perturbations of rho and p from 16 Fourier modes (integer wave vectors in
[1,4]^3, phases U[0, 2pi), numpy PCG64 seed 0).  Zero-gradient outflow
(Neumann) on all six faces, AUSM flux, RK2.
"""
from __future__ import annotations

import math

import numpy as np

from . import _ffi as F
from .solver import GridSpec, cell_average, euler_neumann


def fourier_modes(n=16, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.integers(1, 5, size=(n, 3))
    phase = rng.uniform(0.0, 2 * math.pi, size=n)
    return k.astype(np.float64), phase


def riemann3d_ic(modes, amp=0.01, x0=0.5, left=(1.0, 1.0), right=(0.125, 0.1), gamma=1.4):
    k, phase = modes
    nm = len(phase)

    def f(x):  # x: (3, n) -> conserved (5, n); same arithmetic as the oracle's IC kind 5
        pert = np.zeros(x.shape[1])
        for m in range(nm):
            arg = phase[m] + 2 * math.pi * k[m, 0] * x[0]
            arg = arg + 2 * math.pi * k[m, 1] * x[1]
            arg = arg + 2 * math.pi * k[m, 2] * x[2]
            pert = pert + np.sin(arg)
        fac = 1.0 + amp * pert / nm
        is_left = x[0] < x0
        rho = np.where(is_left, left[0], right[0]) * fac
        p = np.where(is_left, left[1], right[1]) * fac
        q = np.zeros((5, x.shape[1]))
        q[3] = rho
        q[4] = p / (gamma - 1.0) + 0.5 * rho * 0.0
        return q

    return f


def riemann3d_spec(base_level=6, extra=2, radius=0.25) -> GridSpec:
    return GridSpec(3, [0.0, 0.0, 0.0], [1.0, 1.0, 1.0], base_level,
                    refine=[([0.5, 0.5, 0.5], radius, base_level + extra)])


def riemann3d_oracle_ic(modes, amp=0.01):
    """The same initial condition as an oracle IC_RIEMANN3D_PERTURBED parameter block."""
    k, phase = modes
    ic = [0.5, 1.0, 1.0, 0.125, 0.1, amp, float(len(phase)), 0.0]
    for m in range(len(phase)):
        ic += [k[m, 0], k[m, 1], k[m, 2], phase[m]]
    return ic


def riemann3d_conditions(nd=3):
    return [euler_neumann() for _ in range(2 * nd)]


# ---------------------------------------------------------------------------
# Ensemble of independent 2D isentropic vortices (batched workload).
# ---------------------------------------------------------------------------
def vortex_ic(beta, cx, cy, u=1.0, v=1.0, gamma=1.4):
    """hom3's isentropic vortex (euler/initial_conditions.hpp:14-39) with the
    strength and centre as parameters (hom3 fixes beta = 5, centre (-5, -5))."""
    def f(x):
        dx, dy = x[0] - cx, x[1] - cy
        r2 = dx * dx + dy * dy
        e1 = np.exp(1 - r2)
        e2 = np.exp(2 * (1 - r2))
        uu = u - beta * e1 * dy / (2 * math.pi)
        vv = v + beta * e1 * dx / (2 * math.pi)
        rho = (1 - ((gamma - 1) * beta ** 2 * e2) / (16 * gamma * math.pi ** 2)) ** (1 / (gamma - 1))
        p = rho ** gamma
        q = np.empty((4, x.shape[1]))
        q[0], q[1], q[2] = rho * uu, rho * vv, rho
        q[3] = p / (gamma - 1.0) + 0.5 * rho * (uu * uu + vv * vv)
        return q
    return f


def ensemble_members(n=256, seed=3, nmin=32, nmax=512, patch_max=0.3, h=10.0 / 512):
    """Per-instance parameters: grid nx x ny in U{nmin..nmax}^2 embedded in a
    square root cell at level ceil(log2(max(nx, ny))) with a box domain, a
    refinement patch (+1 level disc) covering U[0, patch_max] of the box, and a
    vortex of strength U[1, 5] centred uniformly in the box."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        nx, ny = (int(v) for v in rng.integers(nmin, nmax + 1, size=2))
        level = int(math.ceil(math.log2(max(nx, ny))))
        frac = float(rng.uniform(0.0, patch_max))
        area = frac * nx * ny * h * h
        pr = math.sqrt(area / math.pi)
        pc = (float(rng.uniform(0, nx * h)), float(rng.uniform(0, ny * h)))
        beta = float(rng.uniform(1.0, 5.0))
        cc = (float(rng.uniform(0, nx * h)), float(rng.uniform(0, ny * h)))
        out.append(dict(nx=nx, ny=ny, level=level, h=h, patch=(pc, pr), patch_frac=frac, beta=beta, centre=cc))
    return out


def ensemble_member_tables(m):
    """Grid tables of one ensemble member from the library's builder."""
    from .solver import GridSpec, build_tables, edge, square
    h, nx, ny, level = m["h"], m["nx"], m["ny"], m["level"]
    side = h * 2 ** level
    (px, py), pr = m["patch"]
    refine = [([px, py], pr, level + 1)] if pr > 0.5 * h else []
    spec = GridSpec(2, [0.0, 0.0], [side, side], level, refine=refine)
    lx, ly = nx * h, ny * h
    eps = side * 1e-15
    geoms = [edge([eps, 0], [1, 0]), edge([lx - eps, 0], [-1, 0]), edge([0, eps], [0, 1]), edge([0, ly - eps], [0, -1])]
    dom = square([0.5 * lx, 0.5 * ly], [lx, ly])
    return build_tables(spec, geoms, dom, 2)


# ---------------------------------------------------------------------------
# Conjugate heat transfer: a CNS channel over a heat-conducting solid.
# ---------------------------------------------------------------------------
def cht_setup(level=9, side=4.0, fluid_rows=128, solid_rows=64, kappa=10.0, seed=1, amp=0.1, Minfty=0.2,
              ReInfty=100.0):
    """Fluid (CNS) block of 2^level x fluid_rows cells above a solid (heat)
    block of 2^level x solid_rows cells, both in one square root cell
    [0, side]^2 at `level`, split by domain predicates as in hom3's coupled
    test (coupled_cns_heat_test.cpp:93-95,139-141).  Fluid: hom3's free
    stream at Minfty (quantities of cns/quantities.hpp), inflow left, outflow
    right, zero-gradient top; solid: adiabatic (zero heat flux) outside the
    interface; interface conditions with conductivity ratio kappa =
    k_solid / k_fluid.  Solid initial temperature T_inf (1 + amp f), f a
    16-mode smooth field (integer wave numbers 1..4, PCG64 `seed`) scaled to
    max |f| = 1.  Returns a dict with both solvers' tables, conditions,
    partner cells and initial states."""
    from .solver import (GridSpec, Condition, build_tables, cell_average, edge, partner_cells, square)
    h = side / 2 ** level
    eps = side * 1e-15
    y0 = solid_rows * h
    y1 = y0 + fluid_rows * h
    spec = GridSpec(2, [0.0, 0.0], [side, side], level)
    # fluid: left, right, top, interface
    gf = [edge([eps, 0], [1, 0]), edge([side - eps, 0], [-1, 0]), edge([0, y1 - eps], [0, -1]), edge([0, y0 + eps], [0, 1])]
    tf = build_tables(spec, gf, square([0.5 * side, 0.5 * (y0 + y1)], [side, y1 - y0]), 2)
    # solid: left, right, bottom, interface
    gs = [edge([eps, 0], [1, 0]), edge([side - eps, 0], [-1, 0]), edge([0, eps], [0, 1]), edge([0, y0 - eps], [0, -1])]
    ts = build_tables(spec, gs, square([0.5 * side, 0.5 * y0], [side, y0]), 2)
    gm1 = 0.4
    T_inf = 1.0 / (1 + 0.5 * gm1 * Minfty * Minfty)           # euler/quantities.hpp:131-133
    rho_inf = T_inf ** (1 / gm1)
    u_inf = Minfty * math.sqrt(T_inf)
    p_inf = T_inf ** (1.4 / gm1) / 1.4
    fs = [u_inf, 0.0, rho_inf, p_inf]
    cf = [Condition(F.BC_CNS_INFLOW, fs), Condition(F.BC_CNS_OUTFLOW, fs), Condition(F.BC_EULER_NEUMANN),
          Condition(F.BC_CPL_CNS_HEAT, [kappa])]
    cs = [Condition(F.BC_HEAT_NEUMANN, [0.0]), Condition(F.BC_HEAT_NEUMANN, [0.0]), Condition(F.BC_HEAT_NEUMANN, [0.0]),
          Condition(F.BC_CPL_HEAT_CNS, [kappa])]
    qf = np.zeros((4, tf["ncells"]))
    fgf = tf["first_ghost"]
    qf[0, :fgf] = rho_inf * u_inf
    qf[2, :fgf] = rho_inf
    qf[3, :fgf] = p_inf / gm1 + 0.5 * rho_inf * u_inf * u_inf
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.integers(1, 5, size=(16, 2)).astype(np.float64)
    ph = rng.uniform(0, 2 * math.pi, size=16)

    def field(x):
        f = np.zeros(x.shape[1])
        for m in range(16):
            f = f + np.sin(2 * math.pi * (k[m, 0] * x[0] / side + k[m, 1] * x[1] / side) + ph[m])
        return f

    fgs = ts["first_ghost"]
    xs = ts["x_center"][:, :fgs]
    fmax = np.abs(field(xs)).max()
    qs = np.zeros((1, ts["ncells"]))
    qs[:, :fgs] = cell_average(lambda x: (T_inf * (1 + amp * field(x) / fmax))[None, :], xs, ts["length"][:fgs], 2)
    return dict(tables_fluid=tf, tables_solid=ts, conditions_fluid=cf, conditions_solid=cs,
                partners_fluid=partner_cells(tf, ts), partners_solid=partner_cells(ts, tf), q_fluid=qf, q_solid=qs,
                props=dict(Minfty=Minfty, ReInfty=ReInfty, Pr0=0.72, cfl=0.4, cfl_viscous=0.4), T_inf=T_inf, h=h)


# ---- advection (advection/tests/advection_fv_solver_test.cpp) ----
def rotation_velocity(x, u_mag=0.5, centre=(0.5, 0.5)):
    """radial_velocity of advection_fv_solver_test.cpp:69-85 (a rotation about
    the centre), written as the test writes it, for points x [2][n]."""
    c0, c1 = centre
    radius = np.sqrt((x[0] - c0) ** 2 + (x[1] - c1) ** 2)
    angle = 0.5 * math.pi - np.arccos((x[0] - c0) / radius)
    v0 = np.abs(radius * u_mag * np.sin(angle + 0.5 * math.pi))
    v1 = np.abs(radius * u_mag * np.cos(angle + 0.5 * math.pi))
    v0 = np.where(x[1] - c1 > 0.0, -v0, v0)
    v1 = np.where(x[0] - c0 < 0.0, -v1, v1)
    return np.stack([v0, v1])


def disc_ic(centre=(0.25, 0.5), radius=0.08, q_in=1.0, q_out=0.1):
    """constant_ic of advection_fv_solver_test.cpp:106-115: q_in inside the disc, q_out outside."""
    def f(x):
        r = np.sqrt((x[0] - centre[0]) ** 2 + (x[1] - centre[1]) ** 2)
        return np.where(r - radius > 0.0, q_out, q_in)[None, :]
    return f
