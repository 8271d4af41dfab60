"""h3c_write_vtk: hom3's write_domain (solver.hpp:328-376) in its legacy
binary VTK layout (io/vtk.hpp), checked field by field against the oracle."""
import numpy as np
import pytest

import cases
import vtk_legacy
from oracle import h3o

pytestmark = pytest.mark.gpu

INVALID_SIND = 2147483647  # an internal cell's bc index, written as is (a valid Ind)


def _expected_vertices(t, nd):
    xc, ln = t["x_center"], t["length"]
    rel = np.array([[1 if (v >> d) & 1 else -1 for d in range(nd)] for v in range(1 << nd)], np.float64)
    return xc.T[:, None, :] + 0.5 * ln[:, None, None] * rel[None, :, :]  # [n][2^nd][nd]


def _write_and_read(o, g, tmp_path, node=True):
    t = o.tables()
    g.write_vtk(tmp_path / "domain", t["node"] if node else None)
    return t, vtk_legacy.read(tmp_path / "domain.vtk")


def _check_mesh(t, f, nd):
    assert f["header"] == ["# vtk DataFile Version 2.0", "HOM3 legacy vtk Output ", "BINARY",
                           "DATASET UNSTRUCTURED_GRID"]
    n = t["ncells"]
    verts = _expected_vertices(t, nd)
    uniq = np.unique(verts.reshape(-1, nd), axis=0)  # lexicographic: x, then y, then z
    pts = f["points"]
    assert pts.shape[0] == uniq.shape[0]
    assert np.array_equal(pts[:, :nd], uniq.astype(np.float32))
    if nd == 2:
        assert np.all(pts[:, 2] == 0)
    cells = f["cells"]
    assert cells.shape == (n, (1 << nd) + 1) and np.all(cells[:, 0] == 1 << nd)
    assert np.array_equal(pts[cells[:, 1:], :nd], verts.astype(np.float32))
    assert np.all(f["cell_types"] == (8 if nd == 2 else 11))


def _fields(f):
    return dict(f["fields"]), [k for k, _ in f["fields"]]


def _check_common(t, f, nd, q, node=True):
    d, names = _fields(f)
    n, fg = t["ncells"], t["first_ghost"]
    assert np.array_equal(d["locallCellIds"], np.arange(n))
    assert np.array_equal(d["gridNodeIds"], np.where(t["node"] == h3o.INV, -1, t["node"]) if node
                          else np.full(n, -1))
    for p in range(2 * nd):
        nb = t["neighbors"][p]
        want = np.where((nb >= 0) & (nb < n), nb, -1)
        assert np.array_equal(d[f"local_nghbrs_{p}"], want), p
    assert np.array_equal(d["ghost_cell"], np.where(np.arange(n) >= fg, 1, -1))
    bc = t["bc_idx"]
    assert np.array_equal(d["bcIdx"][fg:], bc[fg:])
    assert np.all(d["bcIdx"][:fg] == INVALID_SIND)
    return d, names


def _close(a, b, rtol=2e-6):
    b = np.asarray(b, np.float64)
    return np.abs(a.astype(np.float64) - b).max() <= rtol * max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("nd", [2, 3])
def test_vtk_euler(nd, tmp_path):
    _, (o,) = cases.euler_case("sod", nd=nd, level=5 if nd == 2 else 3, ti=h3o.RK2)
    g = cases.gpu_solver_from_oracle(o)
    o.solve(3)
    g.solve(3)
    t, f = _write_and_read(o, g, tmp_path)
    _check_mesh(t, f, nd)
    o.apply_bcs(0)
    q = o.state(0)
    d, names = _check_common(t, f, nd, q)
    cv = [f"rho_u{i}" for i in range(nd)] + ["rho", "rho_E"]
    pv = ["a", "p"] + [f"u_{i}" for i in range(nd)] + ["M", "e", "T"]
    assert names == ["locallCellIds", "gridNodeIds"] + [f"local_nghbrs_{p}" for p in range(2 * nd)] + \
        ["ghost_cell", "bcIdx"] + cv + pv
    for v, name in enumerate(cv):
        assert _close(d[name], q[v]), name
    rho, rhoE = q[nd], q[nd + 1]
    u = q[:nd] / rho
    p = 0.4 * (rhoE - 0.5 * rho * (u * u).sum(axis=0))
    a = np.sqrt(1.4 * p / rho)
    want = {"a": a, "p": p, "M": np.sqrt((u * u).sum(axis=0)) / a, "e": p / 0.4 / rho, "T": 1.4 * p / rho}
    for i in range(nd):
        want[f"u_{i}"] = u[i]
    for k, v in want.items():
        assert _close(d[k], v, 1e-5), k


def test_vtk_cns_vorticity(tmp_path):
    _, (o,) = cases.cns_case("sod", level=5)
    g = cases.gpu_solver_from_oracle(o)
    o.solve(2)
    g.solve(2)
    t, f = _write_and_read(o, g, tmp_path, node=False)
    _check_mesh(t, f, 2)
    o.apply_bcs(0)
    q = o.state(0)
    d, names = _check_common(t, f, 2, q, node=False)
    assert names[-2:] == ["mu", "vorticity"]
    # interior cells: central slopes (solver.hpp:596-623) of rho u and rho, slope_u (cns/physics.hpp:89-94)
    fg = t["first_ghost"]
    nb = t["neighbors"]
    ln = t["length"]

    def slope(v, sd, c):
        return (q[v, nb[2 * sd + 1, c]] - q[v, nb[2 * sd, c]]) / (2 * ln[c])

    c = np.arange(fg)
    rho = q[2, c]

    def slope_u(i, sd):
        return (slope(i, sd, c) * rho - slope(2, sd, c) * q[i, c]) / rho ** 2

    w = slope_u(1, 0) - slope_u(0, 1)
    assert _close(d["vorticity"][:fg], w, 1e-4)
    qq = o.quantities()
    p = 0.4 * (q[3] - 0.5 * q[2] * ((q[:2] / q[2]) ** 2).sum(axis=0))
    T = 1.4 * p / q[2]
    s = qq["sOverTref"]
    assert _close(d["mu"], T ** 1.5 * (1 + s) / (T + s), 1e-5)


def test_vtk_advection_velocity(tmp_path):
    _, (o,) = cases.advection_case(level=5)
    g = cases.gpu_solver_from_oracle(o)
    g.solve(2)
    t, f = _write_and_read(o, g, tmp_path)
    d, names = _fields(f)
    assert names[-3:] == ["q", "u_0", "u_1"]
    u = o.velocity()
    assert np.array_equal(d["u_0"], u[0].astype(np.float32)) and np.array_equal(d["u_1"], u[1].astype(np.float32))
