"""Malformed grid tables are rejected by h3c_set_grid with a named error
before anything reaches the device, and the solver stays usable: the valid
tables set afterwards step to the oracle's result.  hom3 itself asserts these
invariants only in debug builds (ASSERT, misc/error.hpp:27-38) and otherwise
reads out of range; the library returns H3C_E_INVALID instead."""
import numpy as np
import pytest

import cases
import hom3_b200 as hb
from hom3_b200.solver import Condition
from oracle import h3o
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu

INVALID = np.iinfo(np.int64).max  # hom3's invalid cell id (misc/indices.hpp)


def _case():
    _, (o,) = cases.euler_case("sod", nd=2, level=3, ti=h3o.RK2)
    info = o.info()
    t = o.tables()
    conds = [Condition(k, v) for k, v in info["bcs"]]
    props = {k: info[k] for k in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")}
    s = hb.Solver(info["nd"], info["physics"], info["flux"], info["ti"], 0, **props)
    return o, s, t, conds


def _ghost_of_kind(t, fg, n_nbrs):
    """A ghost cell id and the positions of its valid neighbours."""
    nb = t["neighbors"]
    n = nb.shape[1]
    for g in range(fg, n):
        pos = [p for p in range(nb.shape[0]) if 0 <= nb[p, g] < n]
        if len(pos) == n_nbrs:
            return g, pos
    raise AssertionError("no such ghost")


def _mutate(kind, t):
    """A copy of the tables with one defect, and the message the library gives."""
    nb, ln, bc = t["neighbors"].copy(), t["length"].copy(), t["bc_idx"].copy()
    fg, n = t["first_ghost"], nb.shape[1]
    if kind == "neighbour_out_of_range":
        nb[1, 5] = n + 7
        msg = "no neighbour"
    elif kind == "neighbour_missing":
        nb[2, 3] = INVALID
        msg = "no neighbour"
    elif kind == "length_zero":
        ln[4] = 0.0
        msg = "length <= 0"
    elif kind == "ghost_two_neighbours":
        g, pos = _ghost_of_kind(t, fg, 1)
        other = (pos[0] ^ 1)  # the opposite position gets an interior cell too
        nb[other, g] = 0
        msg = "neighbours"
    elif kind == "ghost_linked_to_ghost":
        g, pos = _ghost_of_kind(t, fg, 1)
        nb[pos[0], g] = n - 1 if g != n - 1 else n - 2
        msg = "linked to ghost"
    elif kind == "bc_index_out_of_range":
        bc[fg] = 99
        msg = "bc index"
    else:
        raise ValueError(kind)
    return nb, ln, bc, fg, msg


@pytest.mark.parametrize("kind", ["neighbour_out_of_range", "neighbour_missing", "length_zero",
                                  "ghost_two_neighbours", "ghost_linked_to_ghost", "bc_index_out_of_range"])
def test_malformed_tables_are_rejected_and_the_solver_stays_usable(kind):
    o, s, t, conds = _case()
    nb, ln, bc, fg, msg = _mutate(kind, t)
    with pytest.raises(hb.H3cError, match=msg):
        s.set_grid(nb, t["x_center"], ln, bc, fg, conds, t["subface_cells"])
    # the same handle with the valid tables steps as the oracle does
    s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg, conds, t["subface_cells"])
    s.set_state(o.state(0), 0)
    s.reset_time()
    o.solve(2)
    s.solve(2)
    assert rel_err(s.state(0)[:, :fg], o.state(0)[:, :fg]) <= 1e-12


@pytest.mark.parametrize("sizes", ["no_cells", "first_ghost_zero", "first_ghost_past_the_end"])
def test_bad_sizes_are_rejected(sizes):
    o, s, t, conds = _case()
    nb, xc, ln, bc, fg = t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"]
    if sizes == "no_cells":
        nb, xc, ln, bc, fg = nb[:, :0], xc[:, :0], ln[:0], bc[:0], 0
    elif sizes == "first_ghost_zero":
        fg = 0
    else:
        fg = nb.shape[1] + 1
    with pytest.raises(hb.H3cError, match="bad sizes"):
        s.set_grid(nb, xc, ln, bc, fg, conds, t["subface_cells"])


def test_condition_index_past_the_list_is_rejected():
    """A ghost naming a condition that was not appended (hom3's append_bc
    order, solver.hpp:159-169) is refused, not read past the list."""
    o, s, t, conds = _case()
    with pytest.raises(hb.H3cError, match="bc index"):
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"], conds[:-1],
                   t["subface_cells"])


def test_set_grid_on_many_fresh_handles():
    """Table uploads are ordered before the solver stream's kernels read them:
    many handles created and given tables back to back (as a finite-difference
    loop does) all accept the valid tables and step to the same state."""
    o, _, t, conds = _case()
    info = o.info()
    props = {k: info[k] for k in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")}
    q0, fg, ref = o.state(0), t["first_ghost"], None
    for _ in range(40):
        s = hb.Solver(info["nd"], info["physics"], info["flux"], info["ti"], 0, **props)
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg, conds, t["subface_cells"])
        s.set_state(q0, 0)
        s.reset_time()
        s.solve(1)
        q = s.state(0)[:, :fg]
        if ref is None:
            ref = q
        assert np.array_equal(q, ref)
        del s
