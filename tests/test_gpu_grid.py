"""h3c_grid_build_device: the grid builder's tables computed on the GPU, equal
to the host builder's (and so to hom3's tables where the oracle pins them)
array for array, bit for bit."""
import time

import numpy as np
import pytest

import hom3_b200 as hb
from hom3_b200 import solver as S
from hom3_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _both(spec, geoms, dom=None, dk=0):
    th = hb.build_tables(spec, geoms, dom, dk)
    td = hb.build_tables(spec, geoms, dom, dk, device=True)
    return th, td


def _same(th, td):
    assert th["ncells"] == td["ncells"] and th["first_ghost"] == td["first_ghost"]
    for k in ("neighbors", "x_center", "length", "bc_idx"):
        assert th[k].dtype == td[k].dtype and np.array_equal(th[k], td[k]), k
    if th["subface_cells"] is None:
        assert td["subface_cells"] is None
    else:
        assert np.array_equal(th["subface_cells"], td["subface_cells"])


CASES = {
    "2d_unit_l5": lambda: (S.GridSpec(2, [0, 0], [1, 1], 5), None, 0),
    "3d_unit_l4": lambda: (S.GridSpec(3, [0, 0, 0], [1, 1, 1], 4), None, 0),
    "2d_vortex_l6": lambda: (S.GridSpec(2, [-8, -8], [8, 8], 6), None, 0),
    "2d_refined": lambda: (S.GridSpec(2, [0, 0], [1, 1], 4, refine=[([0.4, 0.55], 0.2, 7)]), None, 0),
    "3d_refined": lambda: (S.GridSpec(3, [0, 0, 0], [1, 1, 1], 3,
                                      refine=[([0.5, 0.5, 0.5], 0.25, 5), ([0.2, 0.8, 0.3], 0.1, 6)]), None, 0),
    "2d_rect_root": lambda: (S.GridSpec(2, [0, 0], [2, 1], 5), None, 0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_build_matches_host(name):
    spec, dom, dk = CASES[name]()
    _same(*_both(spec, spec.cube_boundaries(), dom, dk))


@pytest.mark.parametrize("which", ["flow_past_cube", "solid_cube"])
def test_device_build_with_domain_predicate(which):
    """initialDomain predicates (solver.hpp:882-892) and an extra boundary."""
    spec = S.GridSpec(2, [-7, -7], [7, 7], 8)
    c0, c1, c2 = S.make_cube([-3, 0], [1, 1], 14 / 256)
    dom, dk, extra = (c0, 1, (c1,)) if which == "flow_past_cube" else (c0, 2, (c2,))
    _same(*_both(spec, spec.cube_boundaries() + list(extra), dom, dk))


def test_device_build_cht_split_domain():
    """The conjugate-heat configuration's fluid and solid blocks (square domains, edge boundaries)."""
    spec = S.GridSpec(2, [0.0, 0.0], [4.0, 4.0], 7)
    eps = 4.0 * 1e-9
    y0, y1 = 1.0, 2.0
    gf = [S.edge([eps, 0], [1, 0]), S.edge([4 - eps, 0], [-1, 0]), S.edge([0, y1 - eps], [0, -1]),
          S.edge([0, y0 + eps], [0, 1])]
    _same(*_both(spec, gf, S.square([2.0, 0.5 * (y0 + y1)], [4.0, y1 - y0]), 2))


def test_device_build_headline_tree():
    """The 3D Riemann workload's tree: 64^3 base +2 levels in the r = 0.25 sphere (1.45 M cells)."""
    spec = W.riemann3d_spec()
    t0 = time.perf_counter()
    td = hb.build_tables(spec, spec.cube_boundaries(), device=True)
    t1 = time.perf_counter()
    th = hb.build_tables(spec, spec.cube_boundaries())
    t2 = time.perf_counter()
    _same(th, td)
    print(f"device build {t1 - t0:.3f} s, host build {t2 - t1:.3f} s, {td['ncells']} cells")
