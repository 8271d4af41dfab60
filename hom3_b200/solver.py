"""Python mirror of hom3's Solver interface, running on the C ABI (include/h3c.h).

hom3's drivers use (src/solver/fv/solver.hpp:88-221, utilities.hpp:98-113):
    Solver(solverIdx, properties); set_initial_condition(f); append_bc(bc);
    initialize(); solve(); dt(); dt(value); min_dt(); time(); step(); Q<tag>()
`FvSolver` below offers the same calls; its grid comes from the library's
own builder (h3c_grid_build).  `Solver` is the thin layer over the ABI used
when the caller already has hom3's cell tables (the drop-in path).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from . import _ffi as F
from ._ffi import check, lib

LHS, RHS = 0, 1
INV64 = np.iinfo(np.int64).max
INV32 = np.iinfo(np.int32).max

_DEFAULTS = dict(time_end=1.0, cfl=0.2, cfl_viscous=0.4, gamma=1.4, Rspecific=287.058, T0=273.15, rho0=1.225,
                 Minfty=0.1, ReInfty=100.0, Pr0=0.72, Sutherland0=110.4, diffusivity=1.0, T_ref=273.15,
                 limiter_k=1.0)
# hom3 property names -> desc fields
_PROP_KEYS = {"timeEnd": "time_end", "CFL": "cfl", "CFL_viscous": "cfl_viscous", "gamma": "gamma",
              "Rspecific": "Rspecific", "T0": "T0", "rho0": "rho0", "Minfty": "Minfty", "ReInfty": "ReInfty",
              "Pr0": "Pr0", "Sutherland0": "Sutherland0", "diffusivity": "diffusivity", "T_ref": "T_ref"}


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _lp(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


# ---------------------------------------------------------------------------
# geometry (geometry/implicit.hpp:39-205) and conditions
# ---------------------------------------------------------------------------
def fma_rates():
    """(FP64, FP32) fused multiply-adds per second of the current device (h3c_fma_rates)."""
    a, b = C.c_double(), C.c_double()
    check(lib().h3c_fma_rates(C.byref(a), C.byref(b)))
    return a.value, b.value


class _DeviceArray:
    """A device pointer presented through __cuda_array_interface__ (torch.as_tensor makes a view of it)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _device_view(ptr, shape, typestr):
    import torch
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr), device="cuda")


def _sdf(kind, p, inverted=False) -> F.Sdf:
    s = F.Sdf()
    s.kind = kind
    s.inverted = int(bool(inverted))
    for i, v in enumerate(p):
        s.p[i] = float(v)
    return s


def _pad3(v):
    v = list(v)
    return v + [0.0] * (3 - len(v))


def edge(point, normal) -> F.Sdf:
    return _sdf(F.SDF_EDGE, _pad3(point) + _pad3(normal))


def square(center, lengths, inverted=False) -> F.Sdf:
    return _sdf(F.SDF_SQUARE, _pad3(center) + _pad3(lengths), inverted)


def sphere(center, radius, inverted=False) -> F.Sdf:
    return _sdf(F.SDF_SPHERE, _pad3(center) + [radius], inverted)


def make_cube(x_center, dims, cell_length, tol=0.6):
    """geometry/implicit.hpp:182-205: cube, cube grown by one cell, inverted cube shrunk by tol cells."""
    return (square(x_center, dims), square(x_center, [d + cell_length for d in dims]),
            square(x_center, [d - tol * cell_length for d in dims], inverted=True))


@dataclass
class Condition:
    kind: int
    values: Sequence[float] = ()

    def to_c(self) -> F.Bc:
        b = F.Bc()
        b.kind = self.kind
        for i, v in enumerate(self.values):
            b.v[i] = float(v)
        return b


def euler_neumann(flux=()):
    return Condition(F.BC_EULER_NEUMANN, flux)


def euler_dirichlet(state):
    return Condition(F.BC_EULER_DIRICHLET, state)


def euler_vortex():
    return Condition(F.BC_EULER_VORTEX)


def cns_inflow(pv):
    return Condition(F.BC_CNS_INFLOW, pv)


def cns_outflow(pv):
    return Condition(F.BC_CNS_OUTFLOW, pv)


def cns_adiabatic_noslip():
    return Condition(F.BC_CNS_ADIABATIC_NOSLIP)


def cns_adiabatic_slip():
    return Condition(F.BC_CNS_ADIABATIC_SLIP)


def cns_isothermal_noslip(T):
    return Condition(F.BC_CNS_ISOTHERMAL_NOSLIP, [T])


def heat_dirichlet(T):
    return Condition(F.BC_HEAT_DIRICHLET, [T])


def heat_neumann(q):
    return Condition(F.BC_HEAT_NEUMANN, [q])


def adv_dirichlet(value):
    return Condition(F.BC_ADV_DIRICHLET, [value])


def adv_neumann(flux):
    return Condition(F.BC_ADV_NEUMANN, [flux])


def adv_characteristic():
    return Condition(F.BC_ADV_CHARACTERISTIC)


# ---------------------------------------------------------------------------
# thin solver over the ABI
# ---------------------------------------------------------------------------
class Solver:
    """One h3c solver: tables in the caller's numbering, state columns [nv, n_cells]."""

    def __init__(self, nd=2, physics=F.EULER, flux=F.FLUX_AUSM, time_integration=F.EULER_FORWARD,
                 precision=F.FP64, reconstruction=F.RECON_NONE, **props):
        d = F.Desc()
        d.nd, d.physics, d.flux, d.time_integration, d.precision = nd, physics, flux, time_integration, precision
        d.reconstruction = reconstruction
        vals = dict(_DEFAULTS)
        for k, v in props.items():
            vals[_PROP_KEYS.get(k, k)] = v
        for k, v in vals.items():
            setattr(d, k, float(v))
        self.desc = d
        self.nd, self.physics = nd, physics
        self.nv = 1 if physics in (F.HEAT, F.ADVECTION) else nd + 2
        h = C.c_void_p()
        check(lib().h3c_create(C.byref(d), C.byref(h)))
        self.h = h
        self.n_cells = 0
        self.first_ghost = 0

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().h3c_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def _check(self, rc):
        return check(rc, self.h)

    def set_grid(self, neighbors, x_center, length, bc_idx, first_ghost, conditions: Sequence[Condition],
                 subface_cells=None):
        nb = np.ascontiguousarray(neighbors, np.int64)
        xc = np.ascontiguousarray(x_center, np.float64)
        ln = np.ascontiguousarray(length, np.float64)
        bc = np.ascontiguousarray(bc_idx, np.int32)
        n = ln.shape[0]
        g = F.Grid()
        g.n_cells, g.first_ghost, g.ld = n, int(first_ghost), n
        g.neighbors, g.x_center, g.length = _lp(nb), _dp(xc), _dp(ln)
        g.bc_idx = bc.ctypes.data_as(C.POINTER(C.c_int32))
        arr = (F.Bc * max(1, len(conditions)))()
        for i, c in enumerate(conditions):
            arr[i] = c.to_c()
        g.n_bcs, g.bcs = len(conditions), arr
        if subface_cells is not None and len(subface_cells) and np.asarray(subface_cells).size:
            sub = np.ascontiguousarray(subface_cells, np.int64)
            g.n_subfaces = sub.shape[1]
            g.subface_cells = _lp(sub)
        self._check(lib().h3c_set_grid(self.h, C.byref(g)))
        self.n_cells, self.first_ghost = n, int(first_ghost)
        self._grid = (g, nb, xc, ln, bc, arr)  # the tables h3c_write_vtk is handed again

    def set_state(self, q, which=LHS):
        """q: [nv][n_cells] float64, a numpy array or a CUDA tensor (copied device to device)."""
        if hasattr(q, "is_cuda") and q.is_cuda:
            import torch
            t = q.contiguous()
            assert t.dtype == torch.float64 and tuple(t.shape) == (self.nv, self.n_cells), (t.dtype, t.shape)
            self._check(lib().h3c_set_state(self.h, which, C.cast(t.data_ptr(), C.POINTER(C.c_double)),
                                            self.n_cells))
            return
        q = np.ascontiguousarray(q, np.float64)
        assert q.shape == (self.nv, self.n_cells), q.shape
        self._check(lib().h3c_set_state(self.h, which, _dp(q), self.n_cells))

    def set_velocity(self, u):
        """Advection velocity u(x_center) of every cell, ghosts included: [nd][n_cells]
        (Physics::velocity, advection/physics.hpp:104-106)."""
        u = np.ascontiguousarray(u, np.float64)
        assert u.shape == (self.nd, self.n_cells), u.shape
        self._check(lib().h3c_set_velocity(self.h, _dp(u), self.n_cells))

    def write_vtk(self, fname, node_ids=None):
        """write_domain(fName, solver) (solver.hpp:336-376): conditions applied to
        lhs, then fname + ".vtk" in hom3's legacy binary VTK layout."""
        nid = None
        if node_ids is not None:
            nid = np.ascontiguousarray(node_ids, np.int64)
            assert nid.shape == (self.n_cells,)
        self._check(lib().h3c_write_vtk(self.h, str(fname).encode(), C.byref(self._grid[0]),
                                        _lp(nid) if nid is not None else None))

    def state(self, which=LHS, out=None):
        """The state [nv][n_cells] in caller numbering: a new numpy array, or
        written into `out` (a numpy array or a contiguous float64 CUDA tensor)."""
        if out is not None and hasattr(out, "is_cuda") and out.is_cuda:
            import torch
            assert out.dtype == torch.float64 and tuple(out.shape) == (self.nv, self.n_cells) and out.is_contiguous()
            self._check(lib().h3c_get_state(self.h, which, C.cast(out.data_ptr(), C.POINTER(C.c_double)),
                                            self.n_cells))
            return out
        if out is None:
            out = np.empty((self.nv, self.n_cells), np.float64)
        assert out.shape == (self.nv, self.n_cells) and out.dtype == np.float64 and out.flags.c_contiguous
        self._check(lib().h3c_get_state(self.h, which, _dp(out), self.n_cells))
        return out

    Q = state

    def reset_time(self):
        self._check(lib().h3c_reset_time(self.h))

    def solve(self, nsteps=1):
        self._check(lib().h3c_solve(self.h, nsteps))

    def apply_bcs(self, which=LHS):
        self._check(lib().h3c_apply_bcs(self.h, which))

    def _get(self, fn, ctype=C.c_double):
        v = ctype()
        self._check(fn(self.h, C.byref(v)))
        return v.value

    def dt(self, value: Optional[float] = None):
        """dt() reads, dt(value) forces the next step's dt (solver.hpp:112-115)."""
        if value is not None:
            self._check(lib().h3c_force_dt(self.h, float(value)))
            return None
        return self._get(lib().h3c_dt)

    def force_dt(self, value):
        self._check(lib().h3c_force_dt(self.h, float(value)))

    def min_dt(self):
        return self._get(lib().h3c_min_dt)

    def time(self):
        return self._get(lib().h3c_time)

    def step(self):
        return self._get(lib().h3c_step, C.c_int64)

    def status(self):
        return self._get(lib().h3c_status, C.c_int)

    def stream(self):
        v = C.c_void_p()
        self._check(lib().h3c_get_stream(self.h, C.byref(v)))
        return v.value

    def device_state(self, which=LHS):
        ptr = C.POINTER(C.c_double)()
        ld = C.c_int64()
        self._check(lib().h3c_state_device(self.h, which, C.byref(ptr), C.byref(ld)))
        return C.cast(ptr, C.c_void_p).value, ld.value

    def device_order(self):
        out = np.empty(self.n_cells, np.int64)
        self._check(lib().h3c_device_order(self.h, _lp(out)))
        return out

    def set_option(self, option, value):
        self._check(lib().h3c_set_option(self.h, int(option), int(value)))

    def set_persistent_blocks(self, n):
        """Blocks of the Euler/AUSM stage launch (0: the library's default)."""
        self.set_option(F.OPT_PERSISTENT_BLOCKS, n)

    # ---- stepping by parts (one grid split over several solvers) ----
    def stages(self) -> int:
        """Stages per step (h3c_stages)."""
        v = C.c_int()
        self._check(lib().h3c_stages(self.h, C.byref(v)))
        return v.value

    def solve_stage(self, k):
        """Part k of one step (h3c_solve_stage)."""
        self._check(lib().h3c_solve_stage(self.h, k))

    def stage_input(self, k):
        """Part k's input state as a float64 CUDA tensor view [nv][ld] in the
        internal numbering (h3c_stage_input)."""
        p = C.POINTER(C.c_double)()
        self._check(lib().h3c_stage_input(self.h, k, C.byref(p)))
        _, ld = self.device_state(0)
        return _device_view(C.cast(p, C.c_void_p).value, (self.nv, ld), "<f8")

    def dtmin_device(self):
        """The device int64 part 0 takes the step's dt from (h3c_dtmin_device), as a 1-element CUDA tensor view."""
        p = C.POINTER(C.c_int64)()
        self._check(lib().h3c_dtmin_device(self.h, C.byref(p)))
        return _device_view(C.cast(p, C.c_void_p).value, (1,), "<i8")

    def autotune(self, nsteps=20):
        """Times every applicable stage launch configuration from the current
        state and keeps the fastest (h3c_autotune): (choice, ms per step)."""
        ch, ms = C.c_int(), C.c_double()
        self._check(lib().h3c_autotune(self.h, nsteps, C.byref(ch), C.byref(ms)))
        return ch.value, ms.value

    def kernel_info(self) -> dict:
        """The Euler stage launch in use (h3c_kernel_info)."""
        v = np.zeros(8, np.int64)
        self._check(lib().h3c_kernel_info(self.h, _lp(v), 8))
        return {"halo": int(v[0] == 2), "kernel": ("per_cell", "tile", "halo", "cell", "warp", "tile512")[int(v[0])], "halo_slots": int(v[1]),
                "max_halo": int(v[2]), "mean_halo": v[3] / 1000.0, "blocks_per_sm": int(v[4]), "grid": int(v[5]),
                "smem_bytes": int(v[6]), "tiles": int(v[7])}

    def solve_dt(self, dts):
        """Steps with the given time steps (the frozen-dt forward map)."""
        d = np.ascontiguousarray(dts, np.float64)
        self._check(lib().h3c_solve_dt(self.h, d.size, _dp(d)))

    def adjoint(self, nsteps, dJ_dqN, every=0, out=None):
        """Run nsteps steps (CFL dt) and return (dJ/dq0, dts) for J = <dJ_dqN, q_N>.

        every: checkpoint interval (0: chosen by the library).  dJ_dqN may be a
        numpy array or a float64 CUDA tensor of shape [nv][n_cells]; with a CUDA
        tensor the gradient is returned as one (or written into `out`)."""
        dts = np.empty(nsteps)
        if hasattr(dJ_dqN, "is_cuda") and dJ_dqN.is_cuda:
            import torch
            lam = dJ_dqN.contiguous()
            assert lam.dtype == torch.float64 and tuple(lam.shape) == (self.nv, self.n_cells)
            grad = torch.empty_like(lam) if out is None else out
            self._check(lib().h3c_adjoint(self.h, nsteps, every, C.cast(lam.data_ptr(), C.POINTER(C.c_double)),
                                          C.cast(grad.data_ptr(), C.POINTER(C.c_double)), _dp(dts)))
            return grad, dts
        lam = np.ascontiguousarray(dJ_dqN, np.float64)
        assert lam.shape == (self.nv, self.n_cells)
        grad = np.empty_like(lam) if out is None else out
        self._check(lib().h3c_adjoint(self.h, nsteps, every, _dp(lam), _dp(grad), _dp(dts)))
        return grad, dts

    def launches(self):
        return self._get(lib().h3c_launches, C.c_int64)

    def profile(self, enable=True):
        self._check(lib().h3c_profile(self.h, int(enable)))

    def profile_read(self) -> dict:
        n = len(F.KERNEL_KINDS)
        ms = np.zeros(n)
        cnt = np.zeros(n, np.int64)
        self._check(lib().h3c_profile_read(self.h, _dp(ms), _lp(cnt), n))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(F.KERNEL_KINDS) if cnt[i]}

    def set_partner(self, other: "Solver", partner_cells):
        pc = np.ascontiguousarray(partner_cells, np.int64)
        self._check(lib().h3c_set_partner(self.h, other.h, _lp(pc)))

    def set_periodic(self, partner_cells):
        pc = np.ascontiguousarray(partner_cells, np.int64)
        self._check(lib().h3c_set_periodic(self.h, _lp(pc)))


class Batch(Solver):
    """Independent grids of one solver description advanced together
    (h3c_set_grids): one launch per stage over all instances, per-instance
    dt / time / step.  State arrays are the instances' cells concatenated."""

    def set_grids(self, tables: Sequence[dict], conditions: Sequence[Sequence[Condition]]):
        keep = []
        grids = (F.Grid * len(tables))()
        for k, (t, conds) in enumerate(zip(tables, conditions)):
            nb = np.ascontiguousarray(t["neighbors"], np.int64)
            xc = np.ascontiguousarray(t["x_center"], np.float64)
            ln = np.ascontiguousarray(t["length"], np.float64)
            bc = np.ascontiguousarray(t["bc_idx"], np.int32)
            arr = (F.Bc * max(1, len(conds)))()
            for i, c in enumerate(conds):
                arr[i] = c.to_c()
            g = grids[k]
            n = ln.shape[0]
            g.n_cells, g.first_ghost, g.ld = n, int(t["first_ghost"]), n
            g.neighbors, g.x_center, g.length = _lp(nb), _dp(xc), _dp(ln)
            g.bc_idx = bc.ctypes.data_as(C.POINTER(C.c_int32))
            g.n_bcs, g.bcs = len(conds), arr
            sub = t.get("subface_cells")
            if sub is not None and np.asarray(sub).size:
                sub = np.ascontiguousarray(sub, np.int64)
                g.n_subfaces, g.subface_cells = sub.shape[1], _lp(sub)
                keep.append(sub)
            keep += [nb, xc, ln, bc, arr]
        self._check(lib().h3c_set_grids(self.h, len(tables), grids))
        self.sizes = [int(t["ncells"]) for t in tables]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        self.n_cells = int(self.offsets[-1])
        self.first_ghost = sum(int(t["first_ghost"]) for t in tables)
        self.n_instances = len(tables)

    def instance_state(self, q, k):
        return q[:, self.offsets[k]:self.offsets[k + 1]]

    def instances(self):
        n = self.n_instances
        dt, tm, st = np.empty(n), np.empty(n), np.empty(n, np.int64)
        self._check(lib().h3c_instances(self.h, _dp(dt), _dp(tm), _lp(st)))
        return dt, tm, st



def couple_cht(Tr0, cns: Solver, heat: Solver):
    """coupling::apply(Tr0, cns, heat) -- coupling.hpp:52-63."""
    check(lib().h3c_couple_cht(cns.h, heat.h, float(Tr0)), cns.h)


def cht_solve(Tr0, cns: Solver, heat: Solver, nsteps: int):
    """nsteps of coupling::apply(Tr0, cns, heat) + cns.solve() + heat.solve()
    (coupled_cns_heat_test.cpp:235-248), replayed as one CUDA graph."""
    check(lib().h3c_cht_solve(cns.h, heat.h, float(Tr0), int(nsteps)), cns.h)


def cht_adjoint(Tr0, cns: Solver, heat: Solver, nsteps: int, dJ_dqN, dJ_dTN, every: int = 0):
    """Adjoint of nsteps of the coupled loop (h3c_cht_solve) from the current
    states: returns (dJ/dq0 fluid, dJ/dT0 solid, dts [2][nsteps]) for
    J = <dJ_dqN, q_N> + <dJ_dTN, T_N>, time steps frozen."""
    lf = np.ascontiguousarray(dJ_dqN, np.float64)
    lt = np.ascontiguousarray(dJ_dTN, np.float64)
    assert lf.shape == (cns.nv, cns.n_cells) and lt.shape == (heat.nv, heat.n_cells)
    gf, gt, dts = np.empty_like(lf), np.empty_like(lt), np.empty((2, nsteps))
    check(lib().h3c_cht_adjoint(cns.h, heat.h, float(Tr0), int(nsteps), int(every), _dp(lf), _dp(lt), _dp(gf), _dp(gt),
                                _dp(dts)), cns.h)
    return gf, gt, dts


def couple_equal(a: Solver, b: Solver):
    """coupling::apply(s1, s2) -- coupling.hpp:66-73."""
    check(lib().h3c_couple_equal(a.h, b.h), a.h)


# ---------------------------------------------------------------------------
# grids from the library's builder
# ---------------------------------------------------------------------------
@dataclass
class GridSpec:
    """hom3 grid properties: root cell and MinLevel level (grid/helpers.hpp:163-179).
    refine: EXTENSION (not in hom3) -- [(center, radius, level), ...] spheres."""
    nd: int
    xmin: Sequence[float]
    xmax: Sequence[float]
    level: int
    refine: Sequence = ()

    def desc(self, domain=None, domain_kind=0, bc_geoms=()) -> F.GridDesc:
        d = F.GridDesc()
        d.nd = self.nd
        for i in range(self.nd):
            d.xmin[i], d.xmax[i] = self.xmin[i], self.xmax[i]
        d.min_level = self.level
        d.n_refine = len(self.refine)
        for k, (c, r, lvl) in enumerate(self.refine):
            for i, v in enumerate(c):
                d.refine_center[k][i] = v
            d.refine_radius[k] = r
            d.refine_level[k] = lvl
        d.domain_kind = domain_kind
        if domain is not None:
            d.domain = domain
        d.n_bcs = len(bc_geoms)
        for i, g in enumerate(bc_geoms):
            d.bc_geom[i] = g
        return d

    def cube_boundaries(self):
        arr = (F.Sdf * 6)()
        n = lib().h3c_cube_boundaries(C.byref(self.desc()), arr)
        if n < 0:
            check(n)
        return [arr[i] for i in range(n)]

    @property
    def root_length(self):
        return max(self.xmax[i] - self.xmin[i] for i in range(self.nd))

    def cell_length_at_level(self, level):
        return self.root_length / 2.0 ** level


def build_tables(spec: GridSpec, bc_geoms, domain=None, domain_kind=0, device=False) -> dict:
    """Run the library's grid builder -- on the host, or on the GPU with
    device=True (same tables) -- and copy its tables out as numpy arrays."""
    h = C.c_void_p()
    build = lib().h3c_grid_build_device if device else lib().h3c_grid_build
    check(build(C.byref(spec.desc(domain, domain_kind, bc_geoms)), C.byref(h)))
    try:
        v = F.Grid()
        check(lib().h3c_grid_view(h, C.byref(v)))
        n, nd = v.n_cells, spec.nd
        nb = np.ctypeslib.as_array(v.neighbors, shape=(2 * nd * n,)).reshape(2 * nd, n).copy()
        xc = np.ctypeslib.as_array(v.x_center, shape=(nd * n,)).reshape(nd, n).copy()
        ln = np.ctypeslib.as_array(v.length, shape=(n,)).copy()
        bc = np.ctypeslib.as_array(v.bc_idx, shape=(n,)).copy()
        sub = None
        if v.n_subfaces > 0:
            k = 1 << (nd - 1)
            sub = np.ctypeslib.as_array(v.subface_cells, shape=(k * v.n_subfaces,)).reshape(k, v.n_subfaces).copy()
        return dict(neighbors=nb, x_center=xc, length=ln, bc_idx=bc, first_ghost=v.first_ghost, ncells=n,
                    subface_cells=sub)
    finally:
        lib().h3c_grid_free(h)


def cell_average(f: Callable, x_center: np.ndarray, length: np.ndarray, nd: int) -> np.ndarray:
    """quadrature::integrate / volume (quadrature.hpp:43-74, solver.hpp:980-992):
    mean of f over the 2^nd Gauss points (+-1/sqrt(3)), vectorised over cells."""
    gp = 1 / math.sqrt(3)
    acc = None
    for k in range(1 << nd):
        rel = np.array([(1.0 if (k >> d) & 1 else -1.0) * gp for d in range(nd)])[:, None]
        x = x_center + (0.5 * length)[None, :] * rel
        v = np.asarray(f(x), np.float64)
        acc = v if acc is None else acc + v
    vol = length.copy()
    for _ in range(1, nd):
        vol = length * vol
    return acc * vol / float(1 << nd) / vol


def periodic_partners(tables: dict, spec: GridSpec) -> np.ndarray:
    """EXTENSION (not in hom3): for each ghost of a full-box uniform grid, the
    interior cell on the opposite face (wrap-around)."""
    nd, fg, n = spec.nd, tables["first_ghost"], tables["ncells"]
    xc, ln = tables["x_center"], tables["length"]
    lo = np.array([spec.xmin[i] for i in range(nd)])
    L = spec.root_length
    h = ln[:fg].min()
    idx = np.floor((xc[:, :fg] - lo[:, None]) / h).astype(np.int64)
    m = int(round(L / h))
    key = {tuple(idx[:, i]): i for i in range(fg)}
    out = np.full(n - fg, -1, np.int64)
    gi = np.floor((xc[:, fg:] - lo[:, None]) / h).astype(np.int64) % m
    for j in range(n - fg):
        out[j] = key.get(tuple(gi[:, j]), -1)
    return out


def partner_cells(tables_self: dict, tables_other: dict) -> np.ndarray:
    """Coupling partners (coupling.hpp:24-39): the other solver's cell whose
    centre is the ghost's position (both grids from the same root and level)."""
    fg, n = tables_self["first_ghost"], tables_self["ncells"]
    xo = tables_other["x_center"][:, : tables_other["first_ghost"]]
    key = {tuple(np.round(xo[:, i], 12)): i for i in range(xo.shape[1])}
    xs = tables_self["x_center"][:, fg:]
    out = np.full(n - fg, -1, np.int64)
    for j in range(n - fg):
        out[j] = key.get(tuple(np.round(xs[:, j], 12)), -1)
    return out


class FvSolver(Solver):
    """hom3-style solver: properties, initial condition, boundary conditions,
    initialize(), solve() (solver.hpp:88-145)."""

    def __init__(self, grid: GridSpec, properties: dict, physics=F.EULER, flux=F.FLUX_AUSM,
                 time_integration=F.EULER_FORWARD, precision=F.FP64):
        props = {k: v for k, v in properties.items() if k not in ("initialDomain", "initialCondition", "velocity")}
        super().__init__(grid.nd, physics, flux, time_integration, precision, **props)
        self.grid = grid
        self.initial_domain = properties.get("initialDomain", (None, 0))
        self.initial_condition = properties.get("initialCondition")
        # advection: the "velocity" property, a function of the cell centre (advection/physics.hpp:36-37)
        self.velocity = properties.get("velocity")
        self.bcs: list = []
        self.tables: Optional[dict] = None

    def set_initial_condition(self, f: Callable):
        self.initial_condition = f

    def append_bc(self, geometry: F.Sdf, condition: Condition):
        self.bcs.append((geometry, condition))

    def append_bcs(self, pairs):
        for g, c in pairs:
            self.append_bc(g, c)

    def initialize(self):
        dom, kind = self.initial_domain
        t = build_tables(self.grid, [g for g, _ in self.bcs], dom, kind)
        self.tables = t
        self.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"],
                      [c for _, c in self.bcs], t["subface_cells"])
        if self.physics == F.ADVECTION:
            xc = t["x_center"]
            self.set_velocity(np.stack([np.asarray(self.velocity(xc[:, c]), np.float64)
                                        for c in range(t["ncells"])], axis=1))
        q = np.zeros((self.nv, t["ncells"]))
        fg = t["first_ghost"]
        if self.initial_condition is not None:
            q[:, :fg] = cell_average(self.initial_condition, t["x_center"][:, :fg], t["length"][:fg], self.nd)
        self.set_state(q, LHS)
        self.reset_time()
