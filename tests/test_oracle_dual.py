"""The forward-mode dual-number build of the oracle (Solver<Dual>, which the
GPU's discrete adjoint is compared with) against central finite differences of the
double build: same values bit for bit, derivatives to second order in the
finite-difference step.  Time steps are frozen (forced) in both."""
import numpy as np
import pytest

import cases
from oracle import h3o

BUILDERS = {
    "euler2d_rk2": lambda: cases.euler_case("sod", nd=2, level=4, ti=h3o.RK2),
    "euler_dirichlet_fe": lambda: cases.euler_dirichlet_case(nd=2, level=4),
    "heat3d_fe": lambda: cases.heat_case(level=3),
    "periodic_vortex_rk2": lambda: cases.periodic_vortex_case(level=4),
    "refined_rk2": lambda: cases.refined_case(level=2, fine=3),
    "vortex_muscl_rk3": lambda: cases.periodic_vortex_case(level=4, ti=h3o.SSPRK3, recon=h3o.RECON_MUSCL),
    "cns_walls_fe": lambda: cases.cns_case("walls", level=4),
    "cns_slip_rk2": lambda: cases.cns_case("slip", level=4, ti=h3o.RK2),
    "cns_isothermal_fe": lambda: cases.cns_case("isothermal", level=4),
    "tgv_cns_rk2": lambda: cases.tgv_case(level=3),
    "vortex_muscl_fe": lambda: cases.periodic_vortex_case(level=5, ti=h3o.EULER_FORWARD, recon=h3o.RECON_MUSCL),
}


def frozen_run(build, q, dts):
    _, (s,) = build()
    s.set_state(q)
    for d in dts:
        s.force_dt(d)
        s.solve(1)
    return s.state(0)


@pytest.mark.parametrize("name", sorted(BUILDERS))
def test_dual_oracle_matches_finite_differences(name):
    build = BUILDERS[name]
    _, (o,) = build()
    q1 = cases.smooth_state(o)
    fg = o.first_ghost
    o.set_state(q1)
    dts = []
    for _ in range(4):
        o.solve(1)
        dts.append(o.dt())
    rng = np.random.default_rng(7)
    dq = np.zeros_like(q1)
    dq[:, :fg] = rng.standard_normal((q1.shape[0], fg))
    _, (o2,) = build()
    ds = h3o.DualSolver(o2)
    ds.set_state(q1, dq)
    ds.solve_dt(np.array(dts))
    val, dot = ds.state()
    ref = frozen_run(build, q1, dts)
    assert np.array_equal(val[:, :fg], ref[:, :fg])
    errs = []
    # the limited reconstruction is differentiable only closer to the state than
    # its nearest switch (limiter face, extreme neighbour): smaller steps there
    steps = (1e-7, 1e-8) if "muscl" in name else (1e-4, 1e-5)
    for eps in steps:
        fd = (frozen_run(build, q1 + eps * dq, dts) - frozen_run(build, q1 - eps * dq, dts)) / (2 * eps)
        errs.append(np.abs(dot[:, :fg] - fd[:, :fg]).max() / np.abs(fd[:, :fg]).max())
    if "muscl" in name:
        assert max(errs) < 1e-6, errs
    else:
        assert errs[1] < 1e-7, errs
        assert errs[1] < errs[0] / 30 or errs[1] < 1e-9, errs  # second-order convergence
