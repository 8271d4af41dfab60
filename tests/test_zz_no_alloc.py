"""h3c_min_dt_noalloc: the time step for callers that cannot allocate device
memory (a framework that owns all device memory through its own pool, or a
step controller that must not call cudaMalloc because it synchronises the
device).  Its result must equal the library's h3c_min_dt and the oracle's
min_dt on the same state, call after call, and repeated calls must leave the
device's free memory unchanged.  This file is collected last so a
first-failure run has already run every other test; it also passes alone in
a fresh process."""
import ctypes as C

import numpy as np
import pytest

import cases
from oracle import h3o

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 per-step tolerance of the parity tests
MAX_CELLS = 4 * 1024 * 1024  # the fixed scratch array's limit


def _noalloc(desc, q, ld, n_int, lengths_dev, out, stream):
    import torch
    from hom3_b200 import _ffi as F
    rc = F.lib().h3c_min_dt_noalloc(C.byref(desc), C.c_void_p(q), ld, n_int,
                                    C.c_void_p(lengths_dev.data_ptr()), C.c_void_p(out.data_ptr()),
                                    C.c_void_p(stream))
    F.check(rc)
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("case", ["euler3d", "cns2d", "heat3d"])
def test_noalloc_min_dt_matches_min_dt_and_oracle(case):
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
        ref_lib, ref_oracle = g.min_dt(), o.min_dt()
        assert abs(ref_lib - ref_oracle) <= TOL * ref_oracle
        for _call in range(2):
            q, ld = g.device_state(0)
            got = _noalloc(g.desc, q, ld, n_int, lengths_dev, out, g.stream())
            assert abs(got - ref_lib) <= TOL * ref_lib, (got, ref_lib)
            assert abs(got - ref_oracle) <= TOL * ref_oracle, (got, ref_oracle)
            out.fill_(-1.0)
        o.solve(1)
        g.solve(1)


def test_noalloc_at_the_maximum_size_and_without_allocating():
    """n_cells = 4,194,304 (every partial slot of the scratch written and
    folded) on a synthetic 3D Euler state, against the CFL formula of hom3's
    compute_dt (euler/physics.hpp:182-196) evaluated with numpy; then further
    calls change neither the device's free memory nor torch's allocations."""
    import torch
    from hom3_b200 import _ffi as F
    from hom3_b200.solver import Solver
    rng = np.random.default_rng(3)
    n = MAX_CELLS
    rho = rng.uniform(0.5, 2.0, n)
    u = rng.uniform(-0.5, 0.5, (3, n))
    p = rng.uniform(0.2, 3.0, n)
    h = np.where(rng.random(n) < 0.5, 1 / 256, 1 / 512)
    gamma, cfl = 1.4, 0.4
    q = np.empty((5, n))
    q[:3] = rho * u
    q[3] = rho
    q[4] = p / (gamma - 1) + 0.5 * rho * (u * u).sum(axis=0)
    # compute_dt: cfl h / max_d(|u_d| + a), a = sqrt(gamma p / rho), from the conservative state
    uu = q[:3] / q[3]
    pp = (gamma - 1) * (q[4] - 0.5 * q[3] * (uu * uu).sum(axis=0))
    a = np.sqrt(gamma * pp / q[3])
    ref = float(np.min(cfl * h / (np.abs(uu) + a).max(axis=0)))
    s = Solver(3, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, F.FP64, cfl=cfl, gamma=gamma)
    qd = torch.tensor(q, dtype=torch.float64, device="cuda")
    hd = torch.tensor(h, dtype=torch.float64, device="cuda")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    got = _noalloc(s.desc, qd.data_ptr(), n, n, hd, out, stream)  # first call: set-up
    assert abs(got - ref) <= TOL * ref, (got, ref)
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    for _ in range(5):
        out.fill_(-1.0)
        got = _noalloc(s.desc, qd.data_ptr(), n, n, hd, out, stream)
        assert abs(got - ref) <= TOL * ref, (got, ref)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_rejects_sizes_beyond_its_scratch_and_advection():
    import torch
    from hom3_b200 import _ffi as F
    from hom3_b200.solver import Solver
    s = Solver(3)
    big = MAX_CELLS + 1
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = F.lib().h3c_min_dt_noalloc(C.byref(s.desc), C.c_void_p(dummy.data_ptr()), big, big,
                                    C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), None)
    assert rc == F.E_INVALID
    assert "4194304" in F.last_error(None)
    adv = Solver(2, F.ADVECTION, F.FLUX_UPWIND, F.EULER_FORWARD, F.FP64)
    rc = F.lib().h3c_min_dt_noalloc(C.byref(adv.desc), C.c_void_p(dummy.data_ptr()), 1, 1,
                                    C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), None)
    assert rc == F.E_INVALID
    assert "advection" in F.last_error(None)
