"""The C++ host layer (include/hom3_b200.hpp): hom3's solver test cases
written against it compile (CPU) and run to their end times with physical
states on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "hom3_cases.cpp")
LIBDIR = os.path.join(ROOT, "hom3_b200", "_lib")


def build(tmp_path):
    exe = str(tmp_path / "hom3_cases")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-lhom3_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_cpp_cases_compile_and_link(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_cpp_cases_run(tmp_path):
    exe = build(tmp_path)
    res = subprocess.run([exe, "4"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    rows = [l.split() for l in res.stdout.strip().splitlines()]
    names = [r[0] for r in rows]
    assert names == ["euler_constant_ic", "euler_sod_shock_tube_ic", "euler_problem123_ic", "euler_explosion_ic",
                     "euler_isentropic_vortex_ic", "heat_one_dimensional_dirichlet"]
    ends = {"euler_constant_ic": 0.25, "euler_sod_shock_tube_ic": 0.2, "euler_problem123_ic": 0.15,
            "euler_explosion_ic": 0.25, "euler_isentropic_vortex_ic": 2.0, "heat_one_dimensional_dirichlet": 0.25}
    for name, steps, time, ok in rows:
        assert ok == "1", name
        assert float(time) >= ends[name] - 1e-12 or int(steps) >= 1000, name
