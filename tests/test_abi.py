"""CPU checks of the C ABI library: it loads, exports every entry point that
include/h3c.h declares, and its host grid builder reproduces the oracle's
hom3 tables exactly (no GPU calls)."""
import os
import re

import numpy as np
import pytest

import hom3_b200 as hb
from hom3_b200 import _ffi as F
from hom3_b200 import solver as S
from oracle import h3o

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "h3c.h")).read()
    return sorted(set(re.findall(r"^\s*int\s+(h3c_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = hb.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for name in syms:
        assert hasattr(L, name), name
        assert name in F.SIGNATURES, f"{name} has no ctypes signature"


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(hb.H3cError):
        hb.Solver(2)


@pytest.mark.parametrize("physics,flux", [(F.ADVECTION, F.FLUX_AUSM), (F.EULER, F.FLUX_UPWIND),
                                          (F.HEAT, F.FLUX_UPWIND), (F.CNS, F.FLUX_UPWIND)])
def test_create_rejects_a_flux_of_another_physics(physics, flux):
    """Checked before any CUDA call: advection takes upwind or LLF, upwind is advection's."""
    with pytest.raises(hb.H3cError, match="flux"):
        hb.Solver(2, physics, flux)


def _oracle_tables(nd, lo, hi, level, domain=None, dk=0, extra=()):
    w = h3o.World(nd, lo, hi, level=level)
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
    for g in extra:
        bcs.append(h3o.bc(h3o.BC_EULER_NEUMANN, _to_oracle_sdf(g)))
    s = w.add_solver(bcs=bcs, domain=_to_oracle_sdf(domain) if domain is not None else None, domain_kind=dk)
    s.initialize()
    return s.tables()


def _to_oracle_sdf(g):
    s = h3o.Sdf()
    s.kind, s.inverted = g.kind, g.inverted
    for i in range(6):
        s.p[i] = g.p[i]
    return s


CASES = {
    "2d_unit_l4": (2, [0, 0], [1, 1], 4, None, 0, ()),
    "3d_unit_l3": (3, [0, 0, 0], [1, 1, 1], 3, None, 0, ()),
    "2d_vortex_l5": (2, [-8, -8], [8, 8], 5, None, 0, ()),
}


@pytest.mark.parametrize("name", list(CASES) + ["flow_past_cube", "solid_cube"])
def test_builder_matches_oracle_tables(name):
    if name in CASES:
        nd, lo, hi, level, dom, dk, extra = CASES[name]
    else:
        nd, lo, hi, level = 2, [-7, -7], [7, 7], 8
        c0, c1, c2 = S.make_cube([-3, 0], [1, 1], 14 / 256)
        dom, dk, extra = (c0, 1, (c1,)) if name == "flow_past_cube" else (c0, 2, (c2,))
    spec = hb.GridSpec(nd, lo, hi, level)
    t = hb.build_tables(spec, spec.cube_boundaries() + list(extra), dom, dk)
    o = _oracle_tables(nd, lo, hi, level, dom, dk, extra)
    assert t["ncells"] == o["ncells"] and t["first_ghost"] == o["first_ghost"]
    for k in ("neighbors", "x_center", "length", "bc_idx"):
        assert np.array_equal(t[k], o[k]), k


def test_builder_sphere_refinement_is_balanced():
    """EXTENSION: refined tree -- every coarse/fine face is a 2:1 sub-face group
    and the leaves tile the root cell."""
    spec = hb.GridSpec(3, [0, 0, 0], [1, 1, 1], 3, refine=[([0.5, 0.5, 0.5], 0.25, 5)])
    t = hb.build_tables(spec, spec.cube_boundaries())
    fg = t["first_ghost"]
    assert abs((t["length"][:fg] ** 3).sum() - 1.0) < 1e-12
    assert t["subface_cells"] is not None and t["subface_cells"].shape[0] == 4
    lv = np.round(np.log2(1.0 / t["length"][:fg])).astype(int)
    nb = t["neighbors"][:, :fg]
    for p in range(6):
        same = (nb[p] >= 0) & (nb[p] < t["ncells"])
        nbl = np.round(np.log2(1.0 / t["length"][nb[p][same]])).astype(int)
        assert np.all(np.abs(nbl - lv[same]) <= 1)
        grp = nb[p] <= -2
        k = -nb[p][grp] - 2
        fine = t["subface_cells"][:, k]
        assert np.all(lv[fine] == (lv[grp] + 1)[None, :])
