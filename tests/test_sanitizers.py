"""The host code under AddressSanitizer and UndefinedBehaviorSanitizer (on CPU).

hom3 runs its tests under ASan/MSan/TSan build types (CMakeLists.txt:56-72);
compute-sanitizer is closed on the GPU pool here, so the host side is checked
this way: the oracle (oracle/h3o_capi.cpp, the restatement every parity test
rests on) built with -fsanitize=address,undefined and stepped through the
physics, conditions, coupling, refined trees, MUSCL/SSP-RK3 and the dual
numbers; and the library's host grid builder (hom3_b200/csrc/grid_build.cpp)
built the same way and run on uniform, refined and domain-cut grids.  Any
report aborts the child process."""
import os
import shutil
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = ["-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined"]
ENV_SAN = {"ASAN_OPTIONS": "detect_leaks=0:abort_on_error=1", "UBSAN_OPTIONS": "print_stacktrace=1:halt_on_error=1"}


def _gcc_lib(name):
    p = subprocess.run(["g++", f"-print-file-name={name}"], capture_output=True, text=True).stdout.strip()
    return p if os.path.isabs(p) and os.path.exists(p) else None


needs_gcc = pytest.mark.skipif(shutil.which("g++") is None or _gcc_lib("libasan.so") is None,
                               reason="g++ with libasan is not available")


@needs_gcc
def test_oracle_under_asan_ubsan(tmp_path):
    lib = str(tmp_path / "libh3o_san.so")
    subprocess.run(["g++", *SAN, "-std=c++17", "-fPIC", "-ffp-contract=off", "-fopenmp", "-shared", "-o", lib,
                    os.path.join(ROOT, "oracle", "h3o_capi.cpp"), "-L/usr/lib/x86_64-linux-gnu", "-l:libgomp.so.1"],
                   check=True)
    script = textwrap.dedent("""
        import sys
        sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
        import numpy as np
        from oracle import h3o
        import cases
        h3o.set_num_threads(2)
        runs = [cases.refined_case(ti=h3o.RK2, level=2, fine=4)[1][0],
                cases.euler_case("sod", nd=3, level=3, ti=h3o.SSPRK3)[1][0],
                cases.euler_dirichlet_case()[1][0],
                cases.cns_case("sod", level=4, ti=h3o.RK2)[1][0],
                cases.heat_case(level=3)[1][0],
                cases.periodic_vortex_case(level=4, ti=h3o.SSPRK3, recon=h3o.RECON_MUSCL, limiter_k=1.0)[1][0],
                cases.tgv_case(level=3)[1][0],
                cases.advection_case(level=5)[1][0]]
        for s in runs:
            s.solve(2)
            assert np.isfinite(s.state(0)).all()
        w, (cns, heat) = cases.cht_case(level=6, kappa=10.0)
        for _ in range(2):
            h3o.couple_cht(cns, heat, 0.01)
            cns.solve(1)
            heat.solve(1)
        for src in (cases.refined_case(ti=h3o.RK2, level=2, fine=4)[1][0], cases.cns_case("sod", level=4)[1][0]):
            d = h3o.DualSolver(src)
            val = src.state(0)
            d.set_state(val, np.ones_like(val))
            d.solve_dt([src.dt(), src.dt()])
            assert np.isfinite(d.state()[1]).all()
        print("ok")
    """).format(root=ROOT, tests=os.path.join(ROOT, "tests"))
    env = dict(os.environ, H3O_LIB=lib, LD_PRELOAD=_gcc_lib("libasan.so") + ":" + (_gcc_lib("libubsan.so") or ""),
               **ENV_SAN)
    r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]


DRIVER = r"""
#include <cstdio>
#include <string>
#include "h3c.h"
namespace gridb { void set_global_error(const std::string&) {} }
static int build(h3c_grid_desc d) {
  const int nb = h3c_cube_boundaries(&d, d.bc_geom);
  if (nb < 0) return 1;
  d.n_bcs = nb;
  h3c_built_grid b = nullptr;
  if (h3c_grid_build(&d, &b)) return 2;
  h3c_grid v{};
  if (h3c_grid_view(b, &v)) return 3;
  long long bad = 0;
  for (long long c = 0; c < v.first_ghost; ++c) bad += !(v.length[c] > 0);
  h3c_grid_free(b);
  return bad ? 4 : 0;
}
int main() {
  for (int nd = 2; nd <= 3; ++nd) {
    h3c_grid_desc d{};
    d.nd = nd;
    for (int i = 0; i < nd; ++i) { d.xmin[i] = 0; d.xmax[i] = 1; }
    d.min_level = nd == 2 ? 5 : 3;
    if (int rc = build(d)) { std::printf("uniform %d: %d\n", nd, rc); return rc; }
    d.n_refine = 1;
    d.refine_center[0][0] = d.refine_center[0][1] = d.refine_center[0][2] = 0.4;
    d.refine_radius[0] = 0.3;
    d.refine_level[0] = d.min_level + 2;
    if (int rc = build(d)) { std::printf("refined %d: %d\n", nd, rc); return rc; }
    d.domain_kind = 2;  // leaves inside a sphere only
    d.domain.kind = H3C_SDF_SPHERE;
    d.domain.p[0] = d.domain.p[1] = d.domain.p[2] = 0.5;
    d.domain.p[3] = 0.45;
    if (int rc = build(d)) { std::printf("domain %d: %d\n", nd, rc); return rc; }
  }
  std::printf("ok\n");
  return 0;
}
"""


@needs_gcc
def test_host_grid_builder_under_asan_ubsan(tmp_path):
    src = tmp_path / "drive.cpp"
    src.write_text(DRIVER)
    exe = str(tmp_path / "drive")
    r = subprocess.run(["g++", *SAN, "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", exe, str(src),
                        os.path.join(ROOT, "hom3_b200", "csrc", "grid_build.cpp")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    r = subprocess.run([exe], env=dict(os.environ, **ENV_SAN), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]
