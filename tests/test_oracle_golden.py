"""The oracle's tree and grid layer against hom3's own golden vectors.

Fixtures: tests/golden/hierarchical_neighbors.json, extracted by
tests/golden/make_golden.py from hom3's
src/containers/hierarchical/tests/hierarchical_container_test.cpp.
"""
import json
import os

import numpy as np
import pytest

from oracle import h3o
import cases

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "hierarchical_neighbors.json")))


def test_grid_size_3d_level2():
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=2)
    assert w.nnodes() == GOLD["size_3d_level2"] == 73


def test_children_and_positions():
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=2)
    assert [w.child(0, i) for i in range(8)] == GOLD["children_of_0"]
    assert [w.child(1, i) for i in range(8)] == GOLD["children_of_1"]
    for i, c in enumerate(GOLD["children_of_0"]):
        assert w.pos_in_parent(c) == i


def test_leaf_flags():
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=2)
    first = GOLD["first_leaf_3d_level2"]
    for n in range(w.nnodes()):
        assert w.is_leaf(n) == (n >= first)


@pytest.mark.parametrize("nd,level,key", [(3, 2, "neighbors_3d_level2"), (2, 3, "neighbors_2d_level3")])
def test_samelvl_neighbors(nd, level, key):
    w = h3o.World(nd, [0] * nd, [1] * nd, level=level)
    rows = GOLD[key].items() if isinstance(GOLD[key], dict) else GOLD[key]
    checked = 0
    for n, row in rows:
        for p, v in enumerate(row):
            assert w.neighbor(int(n), p) == (h3o.INV if v is None else v), (n, p)
            checked += 1
    assert checked > 40


@pytest.mark.parametrize("nd,level", [(3, 2), (2, 3)])
def test_neighbor_consistency(nd, level):
    """consistency_nghbr_check: hierarchical_container_test.cpp:29-40"""
    w = h3o.World(nd, [0] * nd, [1] * nd, level=level)
    opp = [1, 0, 3, 2, 5, 4]
    for n in range(w.nnodes()):
        for p in range(2 * nd):
            m = w.neighbor(n, p)
            if m != h3o.INV:
                assert w.neighbor(m, opp[p]) == n


def test_cht_cell_counts_match_hom3_capacities():
    """coupled_cns_heat_test.cpp:84,130 size the CNS and heat containers at
    exactly 66308 and 396 cells (leaves + ghosts) for this geometry."""
    w, (cns, heat) = cases.cht_case()
    assert cns.ncells == 66308
    assert heat.ncells == 396


def test_cube_cell_counts():
    """no_solver_cells_with_gc (grid/helpers.hpp:39-42): leaves + 2nd faces of ghosts."""
    for nd, level in ((2, 4), (3, 3)):
        w = h3o.World(nd, [0] * nd, [1] * nd, level=level)
        s = w.add_solver(bcs=cases.neumann_cube(w))
        s.initialize()
        assert s.ncells == 2 ** (nd * level) + 2 * nd * 2 ** (level * (nd - 1))
        assert s.first_ghost == 2 ** (nd * level)
