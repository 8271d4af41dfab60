"""ctypes front-end of the CPU oracle (oracle/h3o.hpp).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() to
check the GPU's result and by the CPU-baseline / reference legs of bench.py.  The shipped
library (hom3_b200) never imports it.

Parity status: the grid/neighbour layer is pinned against hom3's golden
tables; the finite-volume arithmetic is "unpinned by hom3's tests" (hom3's
solver tests carry no numeric assertions) and is checked by known-answer
properties instead.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# H3O_LIB names another build of the same sources (the sanitizer test loads one built with ASan/UBSan)
_LIB_PATH = os.environ.get("H3O_LIB") or os.path.join(_HERE, "_build", "libh3o.so")
INV = np.iinfo(np.int64).max
SINV = np.iinfo(np.int32).max

# physics / flux / time integration / bc / ic kinds (oracle/h3o.hpp)
EULER, CNS, HEAT, ADVECTION = 0, 1, 2, 3
AUSM, LLF, UPWIND = 0, 1, 2  # UPWIND: advection only
VEL_CONSTANT, VEL_ROTATION = 0, 1  # advection velocity fields
EULER_FORWARD, RK2, SSPRK3 = 0, 1, 2  # SSPRK3: EXTENSION (not in hom3)
RECON_NONE, RECON_MUSCL = 0, 1  # MUSCL: EXTENSION (not in hom3)
(BC_EULER_NEUMANN, BC_EULER_DIRICHLET, BC_EULER_VORTEX, BC_CNS_INFLOW, BC_CNS_OUTFLOW,
 BC_CNS_ADIABATIC_NOSLIP, BC_CNS_ADIABATIC_SLIP, BC_CNS_ISOTHERMAL_NOSLIP, BC_HEAT_DIRICHLET,
 BC_HEAT_NEUMANN, BC_CPL_EULER_EULER, BC_CPL_CNS_HEAT, BC_CPL_HEAT_CNS, BC_CPL_HEAT_HEAT,
 BC_PERIODIC, BC_ADV_DIRICHLET, BC_ADV_NEUMANN, BC_ADV_CHARACTERISTIC) = range(18)
(IC_CONSTANT_PV, IC_SHOCK_TUBE, IC_VORTEX, IC_EXPLOSION, IC_CONSTANT_CV,
 IC_RIEMANN3D_PERTURBED, IC_VORTEX_PARAM, IC_TAYLOR_GREEN, IC_DISC) = range(9)
SDF_NONE, SDF_EDGE, SDF_SQUARE, SDF_SPHERE = range(4)


class Sdf(C.Structure):
    _fields_ = [("kind", C.c_int), ("inverted", C.c_int), ("p", C.c_double * 6)]


class BcDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("geom", Sdf), ("v", C.c_double * 8), ("partner", C.c_int)]


class SolverDesc(C.Structure):
    _fields_ = [("physics", C.c_int), ("flux", C.c_int), ("time_integration", C.c_int)] + [
        (n, C.c_double) for n in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty",
                                  "ReInfty", "Pr0", "Sutherland0", "diffusivity", "T_ref", "time_end")
    ] + [("domain_kind", C.c_int), ("domain", Sdf), ("ic_kind", C.c_int), ("ic", C.c_double * 80),
         ("n_bcs", C.c_int), ("bcs", C.POINTER(BcDesc)), ("recon", C.c_int), ("limiter_k", C.c_double),
         ("vel_kind", C.c_int), ("vel", C.c_double * 4)]


class Info(C.Structure):
    _fields_ = [("physics", C.c_int), ("flux", C.c_int), ("ti", C.c_int), ("nd", C.c_int), ("n_bcs", C.c_int)] + [
        (n, C.c_double) for n in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")
    ] + [("bc_kind", C.c_int * 16), ("bc_v", (C.c_double * 8) * 16), ("recon", C.c_int), ("limiter_k", C.c_double)]


def build() -> str:
    """Compile the oracle (make in oracle/) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
        P = C.POINTER
        sig = {
            "h3o_world_create": (vp, [i32, P(dbl), P(dbl), i32]),
            "h3o_world_destroy": (None, [vp]),
            "h3o_world_min_level": (i32, [vp, i32]),
            "h3o_world_refine_sphere": (i32, [vp, P(dbl), dbl, i32]),
            "h3o_grid_nnodes": (i64, [vp]),
            "h3o_grid_neighbor": (i64, [vp, i64, i32]),
            "h3o_grid_child": (i64, [vp, i64, i32]),
            "h3o_grid_is_leaf": (i32, [vp, i64]),
            "h3o_grid_level": (i32, [vp, i64]),
            "h3o_grid_pos_in_parent": (i32, [vp, i64]),
            "h3o_grid_coords": (None, [vp, i64, P(dbl)]),
            "h3o_grid_length": (dbl, [vp, i64]),
            "h3o_grid_root_length": (dbl, [vp]),
            "h3o_cube_boundaries": (i32, [vp, P(Sdf)]),
            "h3o_sdf_eval": (dbl, [i32, P(Sdf), P(dbl)]),
            "h3o_add_solver": (i32, [vp, P(SolverDesc)]),
            "h3o_initialize": (i32, [vp, i32]),
            "h3o_solve": (i32, [vp, i32, i32]),
            "h3o_nv": (i32, [vp, i32]),
            "h3o_ncells": (i64, [vp, i32]),
            "h3o_first_ghost": (i64, [vp, i32]),
            "h3o_get_state": (None, [vp, i32, i32, P(dbl)]),
            "h3o_set_state": (None, [vp, i32, i32, P(dbl)]),
            "h3o_get_tables": (None, [vp, i32, P(i64), P(dbl), P(dbl), P(C.c_int32), P(i64)]),
            "h3o_partner_cells": (i32, [vp, i32, P(i64)]),
            "h3o_velocity": (None, [vp, i32, P(dbl)]),
            "h3o_nsubfaces": (i64, [vp, i32]),
            "h3o_subfaces": (None, [vp, i32, P(i64)]),
            "h3o_dt": (dbl, [vp, i32]),
            "h3o_time": (dbl, [vp, i32]),
            "h3o_step": (i64, [vp, i32]),
            "h3o_min_dt": (dbl, [vp, i32]),
            "h3o_force_dt": (None, [vp, i32, dbl]),
            "h3o_apply_bcs": (None, [vp, i32, i32]),
            "h3o_quantities": (None, [vp, i32, P(dbl)]),
            "h3o_couple_cht": (None, [vp, i32, i32, dbl]),
            "h3o_couple_equal": (None, [vp, i32, i32]),
            "h3o_num_threads": (i32, []),
            "h3o_solver_info": (None, [vp, i32, P(Info)]),
            "h3o_dual_clone": (vp, [vp, i32]),
            "h3o_dual_world_destroy": (None, [vp]),
            "h3o_dual_initialize": (i32, [vp]),
            "h3o_dual_set_state": (None, [vp, P(dbl), P(dbl)]),
            "h3o_dual_get_state": (None, [vp, P(dbl), P(dbl)]),
            "h3o_dual_solve_dt": (None, [vp, i32, P(dbl)]),
            "h3o_dual_ncells": (i64, [vp]),
            "h3o_set_num_threads": (None, [i32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def sdf(kind=SDF_NONE, p=(), inverted=False) -> Sdf:
    s = Sdf()
    s.kind = kind
    s.inverted = int(inverted)
    for i, v in enumerate(p):
        s.p[i] = v
    return s


def edge(point, normal):
    return sdf(SDF_EDGE, list(point) + [0] * (3 - len(point)) + list(normal) + [0] * (3 - len(normal)))


def square(center, lengths, inverted=False):
    return sdf(SDF_SQUARE, list(center) + [0] * (3 - len(center)) + list(lengths) + [0] * (3 - len(lengths)),
               inverted)


def sphere(center, r, inverted=False):
    return sdf(SDF_SPHERE, list(center) + [0] * (3 - len(center)) + [r], inverted)


def make_cube(nd, x_center, dims, cell_length, tol=0.6):
    """geometry/implicit.hpp:182-205: (cube0, cube1 = +1 cell, cube2 = inverted -tol cells)."""
    c0 = square(x_center, dims)
    c1 = square(x_center, [d + cell_length for d in dims])
    c2 = square(x_center, [d - tol * cell_length for d in dims], inverted=True)
    return c0, c1, c2


class Solver:
    """One oracle solver living in a World (grid shared with other solvers)."""

    def __init__(self, world: "World", idx: int):
        self.w, self.idx = world, idx

    @property
    def _h(self):
        return self.w.h

    def initialize(self):
        assert lib().h3o_initialize(self._h, self.idx) == 0

    def solve(self, n=1):
        lib().h3o_solve(self._h, self.idx, n)

    @property
    def nv(self):
        return lib().h3o_nv(self._h, self.idx)

    @property
    def ncells(self):
        return lib().h3o_ncells(self._h, self.idx)

    @property
    def first_ghost(self):
        return lib().h3o_first_ghost(self._h, self.idx)

    def state(self, which=0):
        out = np.empty((self.nv, self.ncells), np.float64)
        lib().h3o_get_state(self._h, self.idx, which, _dp(out))
        return out

    def set_state(self, q, which=0):
        q = np.ascontiguousarray(q, np.float64)
        assert q.shape == (self.nv, self.ncells)
        lib().h3o_set_state(self._h, self.idx, which, _dp(q))

    def tables(self):
        n, nd = self.ncells, self.w.nd
        nb = np.empty((2 * nd, n), np.int64)
        xc = np.empty((nd, n), np.float64)
        ln = np.empty(n, np.float64)
        bc = np.empty(n, np.int32)
        node = np.empty(n, np.int64)
        lib().h3o_get_tables(self._h, self.idx, nb.ctypes.data_as(C.POINTER(C.c_int64)), _dp(xc), _dp(ln),
                             bc.ctypes.data_as(C.POINTER(C.c_int32)), node.ctypes.data_as(C.POINTER(C.c_int64)))
        ns = 1 << (nd - 1)
        nsub = lib().h3o_nsubfaces(self._h, self.idx)
        sub = None
        if nsub > 0:
            flat = np.empty(nsub * ns, np.int64)
            lib().h3o_subfaces(self._h, self.idx, flat.ctypes.data_as(C.POINTER(C.c_int64)))
            sub = np.ascontiguousarray(flat.reshape(nsub, ns).T)
        return dict(neighbors=nb, x_center=xc, length=ln, bc_idx=bc, node=node,
                    first_ghost=self.first_ghost, ncells=n, subface_cells=sub)

    def velocity(self):
        """Advection velocity u(x_center) of every cell, ghosts included: [nd][n_cells]."""
        out = np.empty((self.w.nd, self.ncells), np.float64)
        lib().h3o_velocity(self._h, self.idx, _dp(out))
        return out

    def partner_cells(self):
        n = self.ncells - self.first_ghost
        out = np.empty(n, np.int64)
        lib().h3o_partner_cells(self._h, self.idx, out.ctypes.data_as(C.POINTER(C.c_int64)))
        return out

    def dt(self):
        return lib().h3o_dt(self._h, self.idx)

    def time(self):
        return lib().h3o_time(self._h, self.idx)

    def step(self):
        return lib().h3o_step(self._h, self.idx)

    def min_dt(self):
        return lib().h3o_min_dt(self._h, self.idx)

    def force_dt(self, dt):
        lib().h3o_force_dt(self._h, self.idx, dt)

    def apply_bcs(self, which=0):
        lib().h3o_apply_bcs(self._h, self.idx, which)

    def info(self) -> dict:
        i = Info()
        lib().h3o_solver_info(self._h, self.idx, C.byref(i))
        d = {f: getattr(i, f) for f, _ in Info._fields_[:16]}
        d["bcs"] = [(i.bc_kind[k], list(i.bc_v[k])) for k in range(i.n_bcs)]
        d["recon"], d["limiter_k"] = i.recon, i.limiter_k
        return d

    def quantities(self):
        out = np.empty(8, np.float64)
        lib().h3o_quantities(self._h, self.idx, _dp(out))
        keys = ("T_inf", "rho_inf", "u_inf", "p_inf", "mu_inf", "Re0", "gm1", "sOverTref")
        return dict(zip(keys, out.tolist()))


class World:
    """hom3 grid (CartesianHSP) + the solvers that share it."""

    def __init__(self, nd, xmin, xmax, level=None, max_solvers=2):
        self.nd = nd
        lo = np.asarray(xmin, np.float64)
        hi = np.asarray(xmax, np.float64)
        self.h = lib().h3o_world_create(nd, _dp(lo), _dp(hi), max_solvers)
        if level is not None:
            lib().h3o_world_min_level(self.h, level)
        self.solvers = []

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().h3o_world_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def refine_sphere(self, center, r, max_level):
        c = np.asarray(list(center) + [0] * (3 - len(center)), np.float64)
        lib().h3o_world_refine_sphere(self.h, _dp(c), r, max_level)

    # grid queries (golden neighbour tables)
    def nnodes(self):
        return lib().h3o_grid_nnodes(self.h)

    def neighbor(self, n, pos):
        return lib().h3o_grid_neighbor(self.h, n, pos)

    def child(self, n, pos):
        return lib().h3o_grid_child(self.h, n, pos)

    def is_leaf(self, n):
        return bool(lib().h3o_grid_is_leaf(self.h, n))

    def pos_in_parent(self, n):
        return lib().h3o_grid_pos_in_parent(self.h, n)

    def level(self, n):
        return lib().h3o_grid_level(self.h, n)

    def coords(self, n):
        x = np.zeros(3)
        lib().h3o_grid_coords(self.h, n, _dp(x))
        return x[: self.nd]

    def root_length(self):
        return lib().h3o_grid_root_length(self.h)

    def cell_length_at_level(self, level):
        return self.root_length() / 2.0 ** level

    def cube_boundaries(self):
        arr = (Sdf * 6)()
        n = lib().h3o_cube_boundaries(self.h, arr)
        return [arr[i] for i in range(n)]

    def add_solver(self, physics=EULER, flux=AUSM, time_integration=EULER_FORWARD, *, bcs=(),
                   domain=None, domain_kind=0, ic_kind=IC_CONSTANT_PV, ic=(), **props) -> Solver:
        d, arr = _pack_desc(physics, flux, time_integration, bcs=bcs, domain=domain, domain_kind=domain_kind,
                            ic_kind=ic_kind, ic=ic, **props)
        self._keep = getattr(self, "_keep", []) + [arr]
        idx = lib().h3o_add_solver(self.h, C.byref(d))
        assert idx >= 0, "too many solvers for this grid"
        s = Solver(self, idx)
        self.solvers.append(s)
        return s


def bc(kind, geom, values=(), partner=-1) -> BcDesc:
    b = BcDesc()
    b.kind = kind
    b.geom = geom
    for i, v in enumerate(values):
        b.v[i] = v
    b.partner = partner
    return b


def couple_cht(cns: Solver, heat: Solver, Tr0: float):
    lib().h3o_couple_cht(cns.w.h, cns.idx, heat.idx, Tr0)


def couple_equal(a: Solver, b: Solver):
    lib().h3o_couple_equal(a.w.h, a.idx, b.idx)


def set_num_threads(n: int):
    lib().h3o_set_num_threads(n)


def num_threads() -> int:
    return lib().h3o_num_threads()


class DualSolver:
    """Forward-mode derivative twin of an oracle solver (Solver<Dual>): the
    same tree, description and initial condition; the state carries a
    direction and steps run with given (frozen) time steps, so state() returns
    the state and its directional derivative d q_N / d q_0 . dot."""

    def __init__(self, src: Solver):
        self.h = lib().h3o_dual_clone(src.w.h, src.idx)
        assert lib().h3o_dual_initialize(self.h) == 0
        self.nv = src.nv
        self.n = lib().h3o_dual_ncells(self.h)
        assert self.n == src.ncells

    def __del__(self):
        try:
            lib().h3o_dual_world_destroy(self.h)
        except Exception:
            pass

    def set_state(self, val, dot):
        val = np.ascontiguousarray(val, np.float64)
        dot = np.ascontiguousarray(dot, np.float64)
        assert val.shape == dot.shape == (self.nv, self.n)
        lib().h3o_dual_set_state(self.h, _dp(val), _dp(dot))

    def state(self):
        val = np.empty((self.nv, self.n))
        dot = np.empty((self.nv, self.n))
        lib().h3o_dual_get_state(self.h, _dp(val), _dp(dot))
        return val, dot

    def solve_dt(self, dts):
        d = np.ascontiguousarray(dts, np.float64)
        lib().h3o_dual_solve_dt(self.h, d.size, _dp(d))


def _pack_desc(physics=EULER, flux=AUSM, time_integration=EULER_FORWARD, *, bcs=(), domain=None, domain_kind=0,
               ic_kind=IC_CONSTANT_PV, ic=(), recon=RECON_NONE, limiter_k=1.0, vel_kind=VEL_CONSTANT, vel=(),
               **props):
    d = SolverDesc()
    d.recon, d.limiter_k = recon, float(limiter_k)
    d.vel_kind = vel_kind
    for i, v in enumerate(vel):
        d.vel[i] = v
    defaults = dict(cfl=0.2, cfl_viscous=0.4, gamma=1.4, Rspecific=287.058, T0=273.15, rho0=1.225, Minfty=0.1,
                    ReInfty=100.0, Pr0=0.72, Sutherland0=110.4, diffusivity=1.0, T_ref=273.15, time_end=1.0)
    defaults.update(props)
    d.physics, d.flux, d.time_integration = physics, flux, time_integration
    for k, v in defaults.items():
        setattr(d, k, float(v))
    d.domain_kind = domain_kind
    if domain is not None:
        d.domain = domain
    d.ic_kind = ic_kind
    for i, v in enumerate(ic):
        d.ic[i] = v
    arr = (BcDesc * max(1, len(bcs)))()
    for i, b in enumerate(bcs):
        arr[i] = b
    d.n_bcs = len(bcs)
    d.bcs = arr
    return d, arr
