"""Property-based parity (hypothesis): random small grids, refinement, flux,
time integration and condition mixes, stepped on the GPU through the C ABI
and by the oracle; every step must agree to the per-step parity tolerance.
The draws are derandomised, so a run is reproducible."""
import numpy as np
import pytest
from hypothesis import HealthCheck, assume, given, settings
from hypothesis import strategies as st

import cases
from oracle import h3o
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu
STEPS = 3


@st.composite
def euler_grids(draw):
    nd = draw(st.sampled_from([2, 3]))
    level = draw(st.integers(2, 5 if nd == 2 else 3))
    refine = draw(st.booleans())
    centre = [draw(st.floats(0.3, 0.7)) for _ in range(nd)]
    radius = draw(st.floats(0.15, 0.35))
    ti = draw(st.sampled_from([h3o.EULER_FORWARD, h3o.RK2, h3o.SSPRK3]))
    flux = draw(st.sampled_from([h3o.AUSM, h3o.LLF]))
    kinds = [draw(st.sampled_from(["neumann", "dirichlet"])) for _ in range(2 * nd)]
    ic = draw(st.sampled_from(["sod", "explosion"]))
    split = draw(st.floats(0.3, 0.7))
    return nd, level, refine, centre, radius, ti, flux, kinds, ic, split


def build(nd, level, refine, centre, radius, ti, flux, kinds, ic, split):
    w = h3o.World(nd, [0.0] * nd, [1.0] * nd, level=level)
    if refine:
        w.refine_sphere(centre, radius, level + 2)
    g = w.cube_boundaries()
    state = [0.0] * nd + [1.0, 2.5]  # a Dirichlet state at rest: rho 1, p 1
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, x) if k == "neumann" else h3o.bc(h3o.BC_EULER_DIRICHLET, x, state)
           for k, x in zip(kinds, g)]
    if ic == "sod":
        kind, v = h3o.IC_SHOCK_TUBE, [0, 0, split, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1]
    else:
        kind, v = h3o.IC_EXPLOSION, [split, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1]
    s = w.add_solver(h3o.EULER, flux, ti, bcs=bcs, ic_kind=kind, ic=v, time_end=1.0, **cases.EULER_PROPS)
    s.initialize()
    return w, s


def passes_check_variables(q, nd, gamma=cases.EULER_PROPS["gamma"]):
    """hom3's check_variables on every cell: finite, rho > 0, rho E > 0, p > 0."""
    if not np.isfinite(q).all():
        return False
    rho, E = q[nd], q[nd + 1]
    if not ((rho > 0).all() and (E > 0).all()):
        return False
    p = (gamma - 1.0) * (E - 0.5 * (q[:nd] ** 2).sum(axis=0) / rho)
    return bool((p > 0).all())


@settings(max_examples=60, deadline=None, derandomize=True,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.filter_too_much])
@given(euler_grids())
def test_random_euler_grids_match_the_oracle_step_by_step(params):
    # hom3's LLF dissipation (dx/dt on every face, summed over two or three
    # directions) over-corrects in 2D and 3D, and the reference's own update
    # loses positivity on strong jumps there; the property covers the draws
    # on which the reference's states pass its check_variables (positive
    # density, energy and pressure: euler/physics.hpp:229-239), which the
    # library checks after every step and reports as an error.
    _, probe = build(*params)
    ok = True
    for _ in range(STEPS):
        probe.solve(1)
        ok = ok and passes_check_variables(probe.state(0)[:, :probe.first_ghost], params[0])
    assume(ok)
    w, o = build(*params)
    g = cases.gpu_solver_from_oracle(o, 0)
    fg = o.first_ghost
    for step in range(STEPS):
        o.solve(1)
        g.solve(1)
        e = rel_err(g.state(0)[:, :fg], o.state(0)[:, :fg])
        assert e <= 1e-12 * (step + 1), (params, step, e)
        assert abs(g.dt() - o.dt()) <= 1e-12 * o.dt(), (params, step)
