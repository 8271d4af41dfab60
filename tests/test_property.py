"""Property-based checks of the host-side logic (hypothesis, CPU): the
Morton-range partition of random refined trees covers every interior cell
exactly once, every local face reads a local cell or group, and the exchange
lists pair the same global cells; and the oracle conserves mass, momentum and
energy on random periodic refined trees."""
import numpy as np
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from oracle import h3o


def tree(nd, level, centre, radius, periodic=False):
    w = h3o.World(nd, [0.0] * nd, [1.0] * nd, level=level)
    w.refine_sphere(centre, radius, level + 2)
    kind = h3o.BC_PERIODIC if periodic else h3o.BC_EULER_NEUMANN
    bcs = [h3o.bc(kind, g) for g in w.cube_boundaries()]
    s = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_EXPLOSION,
                     ic=[0.5, 0.5, 0.5, 0.2, 1.0, 1.0, 0.125, 0.1], time_end=1.0, cfl=0.4)
    s.initialize()
    return w, s


grids = st.tuples(st.sampled_from([2, 3]), st.integers(2, 3),
                  st.lists(st.floats(0.25, 0.75), min_size=3, max_size=3), st.floats(0.1, 0.35))


@settings(max_examples=25, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(grids, st.integers(1, 6))
def test_partition_of_random_trees(grid, parts):
    from hom3_b200 import domain
    nd, level, centre, radius = grid
    _, s = tree(nd, level, centre[:nd], radius)
    t = s.tables()
    t["ncells"] = s.ncells
    fg = int(t["first_ghost"])
    parts = min(parts, fg)
    subs = domain.partition(t, parts, nd)
    assert np.array_equal(np.sort(np.concatenate([x.cells for x in subs])), np.arange(fg))
    for x in subs:
        lt, gid = x.tables, x.global_ids()
        nl, fl = lt["ncells"], lt["first_ghost"]
        nsub = 0 if lt["subface_cells"] is None else lt["subface_cells"].shape[1]
        for p in range(2 * nd):
            v = lt["neighbors"][p, :fl]
            plain = (v >= 0) & (v < nl)
            grp = (v <= -2) & (-v - 2 < nsub)
            assert (plain | grp).all()
            assert np.array_equal(gid[v[plain]], t["neighbors"][p, x.cells[plain]])
        for peer, recv in x.recv.items():
            assert np.array_equal(subs[peer].cells[subs[peer].send[x.rank]], gid[recv])


# Periodic conditions pair cells of one level across the domain, so the
# refined region stays clear of the boundary.
periodic_grids = st.sampled_from([2, 3]).flatmap(lambda nd: st.tuples(
    st.just(nd), st.integers(3, 4 if nd == 2 else 3),
    st.lists(st.floats(0.45, 0.55), min_size=3, max_size=3), st.floats(0.05, 0.15)))


@settings(max_examples=15, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(periodic_grids)
def test_oracle_conserves_on_random_periodic_trees(grid):
    nd, level, centre, radius = grid
    _, s = tree(nd, level, centre[:nd], radius, periodic=True)
    fg = s.first_ghost
    vol = s.tables()["length"][:fg] ** nd
    before = (s.state(0)[:, :fg] * vol).sum(axis=1)
    s.solve(3)
    after = (s.state(0)[:, :fg] * vol).sum(axis=1)
    assert np.all(np.abs(after - before) <= 1e-12 * np.abs(before).max())
