"""ctypes bindings of include/h3c.h (libhom3_b200.so).

The library is built in-tree (hom3_b200/build.py) for sm_100a.  Importing this
module fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libhom3_b200.so")

# constants of include/h3c.h
OK, E_INVALID, E_CUDA, E_NONFINITE, E_STATE, E_TIMEOUT, E_NOMEM = 0, -1, -2, -3, -4, -5, -6
EULER, CNS, HEAT, ADVECTION = 0, 1, 2, 3
FLUX_AUSM, FLUX_LLF, FLUX_UPWIND = 0, 1, 2
EULER_FORWARD, RUNGE_KUTTA_2, SSPRK3 = 0, 1, 2
RECON_NONE, RECON_MUSCL = 0, 1
FP64, MIXED = 0, 1
(BC_EULER_NEUMANN, BC_EULER_DIRICHLET, BC_EULER_VORTEX, BC_CNS_INFLOW, BC_CNS_OUTFLOW,
 BC_CNS_ADIABATIC_NOSLIP, BC_CNS_ADIABATIC_SLIP, BC_CNS_ISOTHERMAL_NOSLIP, BC_HEAT_DIRICHLET,
 BC_HEAT_NEUMANN, BC_CPL_EULER_EULER, BC_CPL_CNS_HEAT, BC_CPL_HEAT_CNS, BC_CPL_HEAT_HEAT,
 BC_PERIODIC, BC_ADV_DIRICHLET, BC_ADV_NEUMANN, BC_ADV_CHARACTERISTIC, BC_EXCHANGE) = range(19)
SDF_NONE, SDF_EDGE, SDF_SQUARE, SDF_SPHERE = range(4)
(OPT_TILE_KERNEL, OPT_GRAPHS, OPT_HALO_KERNEL, OPT_PERSISTENT_BLOCKS, OPT_CNS_ADJOINT_DUAL,
 OPT_HALO_SLOTS, OPT_EULER_KERNEL) = 1, 2, 3, 4, 5, 6, 7
STATUS_DT, STATUS_STATE, STATUS_TIMEOUT = 1, 2, 4
KERNEL_KINDS = ("bc", "cfl", "scalar", "stage1", "stage2", "slopes", "copy", "adjoint")


class Desc(C.Structure):
    _fields_ = [("nd", C.c_int), ("physics", C.c_int), ("flux", C.c_int), ("time_integration", C.c_int),
                ("precision", C.c_int)] + [
        (n, C.c_double) for n in ("time_end", "cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0",
                                  "Minfty", "ReInfty", "Pr0", "Sutherland0", "diffusivity", "T_ref")] + [
        ("reconstruction", C.c_int), ("limiter_k", C.c_double)]


class Bc(C.Structure):
    _fields_ = [("kind", C.c_int), ("v", C.c_double * 8)]


class Grid(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("first_ghost", C.c_int64), ("ld", C.c_int64),
                ("neighbors", C.POINTER(C.c_int64)), ("x_center", C.POINTER(C.c_double)),
                ("length", C.POINTER(C.c_double)), ("bc_idx", C.POINTER(C.c_int32)), ("n_bcs", C.c_int),
                ("bcs", C.POINTER(Bc)), ("n_subfaces", C.c_int64), ("subface_cells", C.POINTER(C.c_int64))]


class Sdf(C.Structure):
    _fields_ = [("kind", C.c_int), ("inverted", C.c_int), ("p", C.c_double * 6)]


class GridDesc(C.Structure):
    _fields_ = [("nd", C.c_int), ("xmin", C.c_double * 3), ("xmax", C.c_double * 3), ("min_level", C.c_int),
                ("n_refine", C.c_int), ("refine_center", (C.c_double * 3) * 4), ("refine_radius", C.c_double * 4),
                ("refine_level", C.c_int * 4), ("domain_kind", C.c_int), ("domain", Sdf), ("n_bcs", C.c_int),
                ("bc_geom", Sdf * 16)]


# every entry point declared in include/h3c.h: name -> (restype, argtypes)
_vp, _i64, _i32, _dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
_P = C.POINTER
SIGNATURES = {
    "h3c_create": (_i32, [_P(Desc), _P(_vp)]),
    "h3c_destroy": (_i32, [_vp]),
    "h3c_last_error": (_i32, [_vp, C.c_char_p, C.c_size_t]),
    "h3c_set_grid": (_i32, [_vp, _P(Grid)]),
    "h3c_set_grids": (_i32, [_vp, _i32, _P(Grid)]),
    "h3c_instances": (_i32, [_vp, _P(_dbl), _P(_dbl), _P(_i64)]),
    "h3c_autotune": (_i32, [_vp, _i32, _P(_i32), _P(_dbl)]),
    "h3c_set_state": (_i32, [_vp, _i32, _P(_dbl), _i64]),
    "h3c_get_state": (_i32, [_vp, _i32, _P(_dbl), _i64]),
    "h3c_set_velocity": (_i32, [_vp, _P(_dbl), _i64]),
    "h3c_write_vtk": (_i32, [_vp, C.c_char_p, _P(Grid), _P(_i64)]),
    "h3c_state_device": (_i32, [_vp, _i32, _P(_P(_dbl)), _P(_i64)]),
    "h3c_device_order": (_i32, [_vp, _P(_i64)]),
    "h3c_get_stream": (_i32, [_vp, _P(_vp)]),
    "h3c_sizes": (_i32, [_vp, _P(_i64), _P(_i64), _P(_i32)]),
    "h3c_solve": (_i32, [_vp, _i64]),
    "h3c_stages": (_i32, [_vp, _P(_i32)]),
    "h3c_fma_rates": (_i32, [_P(_dbl), _P(_dbl)]),
    "h3c_solve_stage": (_i32, [_vp, _i32]),
    "h3c_stage_input": (_i32, [_vp, _i32, _P(_P(_dbl))]),
    "h3c_dtmin_device": (_i32, [_vp, _P(_P(_i64))]),
    "h3c_reset_time": (_i32, [_vp]),
    "h3c_apply_bcs": (_i32, [_vp, _i32]),
    "h3c_min_dt": (_i32, [_vp, _P(_dbl)]),
    "h3c_dt": (_i32, [_vp, _P(_dbl)]),
    "h3c_force_dt": (_i32, [_vp, _dbl]),
    "h3c_time": (_i32, [_vp, _P(_dbl)]),
    "h3c_step": (_i32, [_vp, _P(_i64)]),
    "h3c_status": (_i32, [_vp, _P(_i32)]),
    "h3c_set_partner": (_i32, [_vp, _vp, _P(_i64)]),
    "h3c_couple_cht": (_i32, [_vp, _vp, _dbl]),
    "h3c_cht_solve": (_i32, [_vp, _vp, _dbl, _i64]),
    "h3c_cht_adjoint": (_i32, [_vp, _vp, _dbl, _i64, _i64, _P(_dbl), _P(_dbl), _P(_dbl), _P(_dbl), _P(_dbl)]),
    "h3c_couple_equal": (_i32, [_vp, _vp]),
    "h3c_set_periodic": (_i32, [_vp, _P(_i64)]),
    "h3c_solve_dt": (_i32, [_vp, _i64, _P(_dbl)]),
    "h3c_adjoint": (_i32, [_vp, _i64, _i64, _P(_dbl), _P(_dbl), _P(_dbl)]),
    "h3c_launches": (_i32, [_vp, _P(_i64)]),
    "h3c_set_option": (_i32, [_vp, _i32, _i32]),
    "h3c_kernel_info": (_i32, [_vp, _P(_i64), _i32]),
    "h3c_selftest_nr": (_i32, [_P(_dbl), _i64, _P(_dbl), _P(_dbl)]),
    "h3c_min_dt_noalloc": (_i32, [_P(Desc), _vp, _i64, _i64, _vp, _vp, _vp]),
    "h3c_profile": (_i32, [_vp, _i32]),
    "h3c_profile_read": (_i32, [_vp, _P(_dbl), _P(_i64), _i32]),
    "h3c_grid_build": (_i32, [_P(GridDesc), _P(_vp)]),
    "h3c_grid_build_device": (_i32, [_P(GridDesc), _P(_vp)]),
    "h3c_grid_view": (_i32, [_vp, _P(Grid)]),
    "h3c_cube_boundaries": (_i32, [_P(GridDesc), _P(Sdf)]),
    "h3c_grid_free": (_i32, [_vp]),
}

_lib = None


class H3cError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"h3c error {code}: {msg}")
        self.code = code


def lib():
    """Load libhom3_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hom3_b200.build` "
                               "(nvcc, sm_100a); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(1024)
    lib().h3c_last_error(handle, buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc, handle=None):
    if rc != OK:
        raise H3cError(rc, last_error(handle))
    return rc
