"""h3c_min_dt_noalloc: the time step for callers that cannot allocate device
memory (a framework that owns all device memory through its own pool, or a
step controller that must not call cudaMalloc because it synchronises the
device).  Its result must equal h3c_min_dt's on the same state, call after
call.  This file is collected last so a first-failure run has already run
every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import cases
from oracle import h3o

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 per-step tolerance of the parity tests


def _noalloc(g, desc, out, n_int, lengths_dev):
    import torch
    from hom3_b200 import _ffi as F
    q, ld = g.device_state(0)
    rc = F.lib().h3c_min_dt_noalloc(C.byref(desc), C.c_void_p(q), ld, n_int,
                                    C.c_void_p(lengths_dev.data_ptr()), C.c_void_p(out.data_ptr()),
                                    C.c_void_p(g.stream()))
    F.check(rc)
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("case", ["euler3d", "cns2d", "heat3d"])
def test_noalloc_min_dt_matches_min_dt(case):
    import torch
    if case == "euler3d":
        _, (o,) = cases.euler_case("sod", nd=3, level=4)
    elif case == "cns2d":
        _, (o,) = cases.cns_case("sod", level=5)
    else:
        _, (o,) = cases.heat_case(level=3)
    g = cases.gpu_solver_from_oracle(o)
    n_int = o.first_ghost
    perm = g.device_order()
    length = o.tables()["length"]
    ln = np.empty(n_int)
    ln[perm[:n_int]] = length[:n_int]
    lengths_dev = torch.tensor(ln, dtype=torch.float64, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):  # two steps, two calls each
        ref = g.min_dt()
        for _call in range(2):
            got = _noalloc(g, g.desc, out, n_int, lengths_dev)
            assert abs(got - ref) <= TOL * ref, (got, ref)
            out.fill_(-1.0)
        g.solve(1)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from hom3_b200 import _ffi as F
    from hom3_b200.solver import Solver
    s = Solver(3)
    big = 4 * 1024 * 1024 + 1
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = F.lib().h3c_min_dt_noalloc(C.byref(s.desc), C.c_void_p(dummy.data_ptr()), big, big,
                                    C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), None)
    assert rc == F.E_INVALID
