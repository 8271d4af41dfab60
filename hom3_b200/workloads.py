"""Synthetic workloads of the benchmark configurations (seeded; no datasets).

riemann3d_refined: 3D Euler on a hierarchical Cartesian tree -- base level 6
(64^3) on the unit cube, refined +2 levels (to level 8) in the sphere of
radius 0.25 at the centre, 2:1 face balanced.  Initial state: Riemann problem
split at x = 0.5 (left rho = 1, p = 1; right rho = 0.125, p = 0.1; u = 0) as
in hom3's shock_tube (euler/initial_conditions.hpp:380-419), with 1%
perturbations of rho and p from 16 Fourier modes (integer wave vectors in
[1,4]^3, phases U[0, 2pi), numpy PCG64 seed 0).  Zero-gradient outflow
(Neumann) on all six faces, AUSM flux, RK2.
"""
from __future__ import annotations

import math

import numpy as np

from . import _ffi as F
from .solver import GridSpec, cell_average, euler_neumann


def fourier_modes(n=16, seed=0):
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.integers(1, 5, size=(n, 3))
    phase = rng.uniform(0.0, 2 * math.pi, size=n)
    return k.astype(np.float64), phase


def riemann3d_ic(modes, amp=0.01, x0=0.5, left=(1.0, 1.0), right=(0.125, 0.1), gamma=1.4):
    k, phase = modes
    nm = len(phase)

    def f(x):  # x: (3, n) -> conserved (5, n); same arithmetic as the oracle's IC kind 5
        pert = np.zeros(x.shape[1])
        for m in range(nm):
            arg = phase[m] + 2 * math.pi * k[m, 0] * x[0]
            arg = arg + 2 * math.pi * k[m, 1] * x[1]
            arg = arg + 2 * math.pi * k[m, 2] * x[2]
            pert = pert + np.sin(arg)
        fac = 1.0 + amp * pert / nm
        is_left = x[0] < x0
        rho = np.where(is_left, left[0], right[0]) * fac
        p = np.where(is_left, left[1], right[1]) * fac
        q = np.zeros((5, x.shape[1]))
        q[3] = rho
        q[4] = p / (gamma - 1.0) + 0.5 * rho * 0.0
        return q

    return f


def riemann3d_spec(base_level=6, extra=2, radius=0.25) -> GridSpec:
    return GridSpec(3, [0.0, 0.0, 0.0], [1.0, 1.0, 1.0], base_level,
                    refine=[([0.5, 0.5, 0.5], radius, base_level + extra)])


def riemann3d_oracle_ic(modes, amp=0.01):
    """The same initial condition as an oracle IC_RIEMANN3D_PERTURBED parameter block."""
    k, phase = modes
    ic = [0.5, 1.0, 1.0, 0.125, 0.1, amp, float(len(phase)), 0.0]
    for m in range(len(phase)):
        ic += [k[m, 0], k[m, 1], k[m, 2], phase[m]]
    return ic


def riemann3d_conditions(nd=3):
    return [euler_neumann() for _ in range(2 * nd)]
