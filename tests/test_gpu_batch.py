"""Batched independent grids (h3c_set_grids): every instance of a batch must
evolve exactly as the same grid stepped alone, each with its own dt."""
import numpy as np
import pytest

import hom3_b200 as hb
from hom3_b200 import _ffi as F
from hom3_b200 import workloads as W
from hom3_b200.solver import euler_neumann

pytestmark = pytest.mark.gpu


def members(n=6):
    ms = W.ensemble_members(n, seed=11, nmin=12, nmax=40)
    tables = [W.ensemble_member_tables(m) for m in ms]
    states = []
    for m, t in zip(ms, tables):
        fg = t["first_ghost"]
        q = np.zeros((4, t["ncells"]))
        q[:, :fg] = hb.cell_average(W.vortex_ic(m["beta"], *m["centre"]), t["x_center"][:, :fg], t["length"][:fg], 2)
        states.append(q)
    return ms, tables, states


@pytest.mark.parametrize("ti", [F.EULER_FORWARD, F.RUNGE_KUTTA_2])
@pytest.mark.parametrize("precision", [F.FP64, F.MIXED])
def test_batch_matches_single_instances(ti, precision):
    ms, tables, states = members()
    conds = [[euler_neumann() for _ in range(4)] for _ in tables]
    b = hb.Batch(2, F.EULER, F.FLUX_AUSM, ti, precision, cfl=0.4, time_end=1e9)
    b.set_grids(tables, conds)
    b.set_state(np.concatenate(states, axis=1), 0)
    b.reset_time()
    b.solve(7)
    qb = b.state(0)
    dtb, tb, sb = b.instances()
    assert np.all(sb == 7)
    assert len(set(np.round(dtb, 15))) > 1  # instances keep their own time step
    for k, (t, q0) in enumerate(zip(tables, states)):
        s = hb.Solver(2, F.EULER, F.FLUX_AUSM, ti, precision, cfl=0.4, time_end=1e9)
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"], conds[k],
                   t["subface_cells"])
        s.set_state(q0, 0)
        s.reset_time()
        s.solve(7)
        fg = t["first_ghost"]
        assert np.array_equal(b.instance_state(qb, k)[:, :fg], s.state(0)[:, :fg]), k
        assert dtb[k] == s.dt() and tb[k] == s.time()


def test_autotune_keeps_the_state():
    ms, tables, states = members(5)
    conds = [[euler_neumann() for _ in range(4)] for _ in tables]

    def make():
        b = hb.Batch(2, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, F.FP64, cfl=0.4, time_end=1e9)
        b.set_grids(tables, conds)
        b.set_state(np.concatenate(states, axis=1), 0)
        b.reset_time()
        return b

    a, b = make(), make()
    choice, ms_step = a.autotune(4)
    assert 0 <= choice < 10 and ms_step > 0
    a.solve(9)
    b.solve(9)
    # the chosen launch configuration may be the other kernel variant, which
    # rounds differently (FMA placement), so compare to rounding
    qa, qb = a.state(0), b.state(0)
    assert np.max(np.abs(qa - qb)) <= 1e-12 * np.max(np.abs(qb))
    ta, tb = a.instances()[1], b.instances()[1]
    assert np.allclose(ta, tb, rtol=1e-12, atol=0)
    assert np.array_equal(a.instances()[2], b.instances()[2])


KERNEL_OF_CHOICE = ["tile"] * 5 + ["per_cell", "cell", "halo", "halo", "halo", "warp", "tile512"]


def test_autotune_single_tree_sets_the_chosen_kernel():
    """On one refined tree every Euler/AUSM configuration applies; the chosen
    one is the kernel in use afterwards and the state is the untuned one's."""
    import torch
    import cases
    from oracle import h3o
    _, (o,) = cases.refined_case(ti=h3o.RK2, level=3, fine=5)
    a = cases.gpu_solver_from_oracle(o, 0)
    b = cases.gpu_solver_from_oracle(o, 0)
    choice, ms_step = a.autotune(3)
    assert 0 <= choice < len(KERNEL_OF_CHOICE) and ms_step > 0
    info = a.kernel_info()
    assert info["kernel"] == KERNEL_OF_CHOICE[choice], (choice, info)
    if 7 <= choice <= 9:  # the halo-staged kernel at 1-3 persistent blocks per SM
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        assert info["grid"] == min(info["tiles"], (choice - 6) * sms)
    a.solve(4)
    b.solve(4)
    fg = o.first_ghost
    qa, qb = a.state(0)[:, :fg], b.state(0)[:, :fg]
    assert np.max(np.abs(qa - qb)) <= 1e-12 * np.max(np.abs(qb))
    assert a.step() == b.step() == 4


def test_autotune_cns_times_the_tile_kernel_grids_and_the_per_cell_kernel():
    """For CNS the candidates are the tile kernel's grid sizes (0-4) and the
    per-cell kernels (5); the state after tuning is the untuned one's."""
    import cases
    from oracle import h3o
    _, (o,) = cases.tgv_case(level=4, ti=h3o.RK2)
    a = cases.gpu_solver_from_oracle(o, 0)
    b = cases.gpu_solver_from_oracle(o, 0)
    choice, ms_step = a.autotune(3)
    assert 0 <= choice <= 5 and ms_step > 0
    assert a.kernel_info()["kernel"] == ("per_cell" if choice == 5 else "halo")
    a.solve(3)
    b.solve(3)
    fg = o.first_ghost
    qa, qb = a.state(0)[:, :fg], b.state(0)[:, :fg]
    assert np.max(np.abs(qa - qb)) <= 1e-12 * np.max(np.abs(qb))


@pytest.mark.parametrize("ti", [F.EULER_FORWARD, F.RUNGE_KUTTA_2])
def test_cns_batch_matches_single_instances(ti):
    """Batches of compressible Navier-Stokes grids (walls, slip walls,
    isothermal walls with inflow/outflow; different sizes, so each keeps its
    own dt) step in the per-cell CNS kernel exactly as each grid alone in the
    same kernel."""
    import cases
    from oracle import h3o
    from hom3_b200.solver import Condition
    osolvers = [cases.cns_case(name, level=lvl, ti=ti)[1][0]
                for name, lvl in (("walls", 4), ("slip", 5), ("isothermal", 4))]
    info = osolvers[0].info()
    props = {k: info[k] for k in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")}
    tables, conds, states = [], [], []
    for o in osolvers:
        assert all(o.info()[k] == v for k, v in props.items())
        t = dict(o.tables())
        t["ncells"] = t["length"].shape[0]
        tables.append(t)
        conds.append([Condition(k, v) for k, v in o.info()["bcs"]])
        states.append(o.state(0))
    b = hb.Batch(2, F.CNS, F.FLUX_AUSM, ti, F.FP64, **props)
    b.set_grids(tables, conds)
    b.set_state(np.concatenate(states, axis=1), 0)
    b.reset_time()
    b.solve(5)
    qb = b.state(0)
    dtb, tb, sb = b.instances()
    assert np.all(sb == 5)
    assert len(set(np.round(dtb, 15))) > 1
    for k, (t, q0) in enumerate(zip(tables, states)):
        s = hb.Solver(2, F.CNS, F.FLUX_AUSM, ti, F.FP64, **props)
        s.set_option(F.OPT_HALO_KERNEL, 0)  # the per-cell CNS kernel, as in the batch
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"], conds[k],
                   t["subface_cells"])
        s.set_state(q0, 0)
        s.reset_time()
        s.solve(5)
        fg = t["first_ghost"]
        assert np.array_equal(b.instance_state(qb, k)[:, :fg], s.state(0)[:, :fg]), k
        assert dtb[k] == s.dt() and tb[k] == s.time()
