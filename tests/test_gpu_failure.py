"""Failure detection through the C ABI.

hom3 ends a run when dt leaves [1e-300, 1e300] (solution_diverged,
utilities.hpp:74-76, 107-110) and asserts positive density, energy and
pressure in every cell (check_variables, euler/physics.hpp:229-239); for heat
only a non-finite temperature counts (hom3's own heat test starts from T = 0).
Here the device records both while it steps and the next read of the step
scalars returns H3C_E_NONFINITE with a message; h3c_status returns and clears
the bits.
The failures are made on the host: a NaN, a negative density or a negative
pressure written into the state with h3c_set_state.  Nothing faults on the
device."""
import numpy as np
import pytest

import cases
import hom3_b200 as hb
from hom3_b200 import _ffi as F
from oracle import h3o

pytestmark = pytest.mark.gpu


def _euler(ti=h3o.RK2):
    _, (o,) = cases.euler_case("sod", nd=3, level=4, ti=ti)
    return o, cases.gpu_solver_from_oracle(o)


def _expect_nonfinite(call, *words):
    with pytest.raises(F.H3cError) as e:
        call()
    assert e.value.code == F.E_NONFINITE
    for w in words:
        assert w in str(e.value), str(e.value)


def test_healthy_run_reports_nothing():
    o, g = _euler()
    g.solve(5)
    assert np.isfinite(g.dt()) and g.status() == 0


@pytest.mark.parametrize("what", ["nan_density", "negative_density", "negative_pressure"])
@pytest.mark.parametrize("ti", [h3o.EULER_FORWARD, h3o.RK2])
def test_bad_cell_written_mid_run_is_reported(what, ti):
    o, g = _euler(ti)
    g.solve(3)
    assert g.status() == 0
    q = g.state(0)
    c = o.first_ghost // 2
    if what == "nan_density":
        q[3, c] = np.nan
    elif what == "negative_density":
        q[3, c] = -0.5
        q[:3, c] = 0.0
    else:
        q[:3, c] = 0.0
        q[4, c] = -1.0  # rho E < 0: negative pressure (and energy)
    g.set_state(q, 0)
    g.solve(1)
    _expect_nonfinite(g.dt, "check_variables")
    _expect_nonfinite(g.time, "check_variables")  # sticky until read by h3c_status
    flags = g.status()
    assert flags & F.STATUS_STATE
    assert g.status() == 0  # cleared


def test_bad_state_is_reported_at_reset_and_by_min_dt():
    o, g = _euler()
    q = g.state(0)
    q[3, 7] = np.nan
    g.set_state(q, 0)
    g.reset_time()  # initialize's set_dt runs the CFL reduction over the state
    _expect_nonfinite(g.dt, "check_variables")
    assert g.status() & F.STATUS_STATE
    _expect_nonfinite(g.min_dt, "check_variables")
    g.status()


def test_unfused_path_reports_too():
    """hom3's vortex condition rewrites boundary cells, so the time step takes
    the separate CFL reduction (k_cfl) at the start of each step."""
    _, (o,) = cases.euler_case("vortex", level=5, ti=h3o.EULER_FORWARD)
    g = cases.gpu_solver_from_oracle(o)
    g.solve(2)
    assert g.status() == 0
    q = g.state(0)
    q[2, o.first_ghost // 3] = -1.0
    g.set_state(q, 0)
    g.solve(1)
    _expect_nonfinite(g.dt, "check_variables")
    g.status()


def test_heat_nonfinite_temperature_is_reported():
    _, (o,) = cases.heat_case(level=3)
    g = cases.gpu_solver_from_oracle(o)
    g.solve(2)
    assert g.status() == 0  # hom3's heat test has T = 0 cells: not a failure
    q = g.state(0)
    q[0, 5] = np.inf
    g.set_state(q, 0)
    g.solve(1)
    _expect_nonfinite(g.dt, "check_variables")
    assert g.status() & F.STATUS_STATE


def test_dt_out_of_range_is_solution_diverged():
    """A forced dt of 1e301 is outside hom3's bounds: solution_diverged."""
    o, g = _euler()
    g.dt(1e301)
    g.solve(1)
    _expect_nonfinite(g.dt, "solution diverged")
    assert g.status() & F.STATUS_DT


def test_batch_instance_failure_names_the_instance():
    from test_gpu_batch import members
    from hom3_b200.solver import euler_neumann
    ms, tables, states = members(4)
    conds = [[euler_neumann() for _ in range(4)] for _ in tables]
    b = hb.Batch(2, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, F.FP64, cfl=0.4, time_end=1e9)
    b.set_grids(tables, conds)
    q = np.concatenate(states, axis=1)
    b.set_state(q, 0)
    b.reset_time()
    b.solve(2)
    b.instances()
    q = b.state(0)
    off = b.offsets[2]  # caller numbering: instance 2 starts here
    q[2, off + 3] = np.nan
    b.set_state(q, 0)
    b.solve(1)
    _expect_nonfinite(b.instances, "instance 2")
    assert b.status() & F.STATUS_STATE
