"""hom3_b200: B200 (sm_100a) finite-volume hot path of gnzlbg/hom3 behind a C ABI.

The compute path is libhom3_b200.so (CUDA, built by hom3_b200.build); this
package is its Python binding and a mirror of hom3's Solver interface.
"""
from . import _ffi  # noqa: F401
from ._ffi import H3cError, lib  # noqa: F401
from .solver import (Batch, FvSolver, GridSpec, Solver, build_tables, cell_average, cht_adjoint, cht_solve,  # noqa: F401
                     couple_cht, couple_equal, partner_cells, periodic_partners)

__all__ = ["Batch", "FvSolver", "GridSpec", "Solver", "build_tables", "cell_average", "cht_adjoint", "cht_solve", "couple_cht", "couple_equal",
           "partner_cells", "periodic_partners", "H3cError", "lib"]
