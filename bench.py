#!/usr/bin/env python
"""Benchmark: cell-updates/s of the finite-volume step on one B200 per rank.

Workload (N=1): 3D Euler on a hierarchical Cartesian tree, base 64^3 on the
unit cube refined +2 levels inside the sphere r = 0.25 at the centre
(1,448,336 leaf cells), seeded perturbed 3D Riemann problem, zero-gradient
outflow on all faces, AUSM flux, RK2 -- see hom3_b200/workloads.py.  One
"step" is one full time step of the solver (Solver::solve: boundary
conditions, dt, both RK stages) over all leaf cells.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
    python bench.py --impl reference ...   # CPU restatement of hom3, all host threads

N > 1 runs independent replicas of the workload, one per GPU (the single grid
is not domain-decomposed): weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        t0 = time.time()  # wait for the first sample so the timed region is covered
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.05)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        busy = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(xs, ws):
    if ws == 1:
        return list(xs)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(xs), dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def hb_fma_rates():
    from hom3_b200.solver import fma_rates
    return fma_rates()


def build_workload(args):
    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import workloads as W

    spec = W.riemann3d_spec(args.base_level, args.extra_levels)
    # the grid tables from the device builder; the host builder's, timed beside, must be identical
    t0 = time.perf_counter()
    t = hb.build_tables(spec, spec.cube_boundaries(), device=True)
    t1 = time.perf_counter()
    th = hb.build_tables(spec, spec.cube_boundaries())
    t2 = time.perf_counter()
    same = all(np.array_equal(t[k], th[k]) for k in ("neighbors", "x_center", "length", "bc_idx")) and (
        (t["subface_cells"] is None and th["subface_cells"] is None) or
        np.array_equal(t["subface_cells"], th["subface_cells"]))
    args.grid_build = {"device_s": round(t1 - t0, 3), "host_s": round(t2 - t1, 3), "identical": bool(same),
                       "what": "h3c_grid_build_device (kernels + download) vs h3c_grid_build (host), same tables"}
    if not same:
        raise RuntimeError("device and host grid builders disagree")
    fg = t["first_ghost"]
    modes = W.fourier_modes()
    q = np.zeros((5, t["ncells"]))
    q[:, :fg] = hb.cell_average(W.riemann3d_ic(modes), t["x_center"][:, :fg], t["length"][:fg], 3)
    prec = F.MIXED if args.precision == "mixed" else F.FP64
    s = hb.Solver(3, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, prec, cfl=args.cfl, time_end=1e30)
    s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg, W.riemann3d_conditions(),
               t["subface_cells"])
    if getattr(args, "euler_kernel", None) is not None:
        s.set_option(F.OPT_EULER_KERNEL, args.euler_kernel)
    return s, t, q, modes


def oracle_solver(args, threads):
    """The CPU restatement of hom3 (oracle/) set up on the default workload:
    hom3's tree (MinLevel + sphere refinement), conditions and initial state."""
    from oracle import h3o
    from hom3_b200 import workloads as W

    h3o.set_num_threads(threads)
    w = h3o.World(3, [0, 0, 0], [1, 1, 1], level=args.base_level)
    w.refine_sphere([0.5, 0.5, 0.5], 0.25, args.base_level + args.extra_levels)
    bcs = [h3o.bc(h3o.BC_EULER_NEUMANN, g) for g in w.cube_boundaries()]
    s = w.add_solver(h3o.EULER, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_RIEMANN3D_PERTURBED,
                     ic=W.riemann3d_oracle_ic(W.fourier_modes()), time_end=1e30, cfl=args.cfl)
    s.initialize()
    return w, s


def cpu_oracle_run(args, steps_budget_s=15.0, max_steps=None, threads=None):
    """Times the oracle on the default workload: one warm-up step, one step
    that sizes the sample to about steps_budget_s, then the timed sample.
    Returns a dict (value in cell-updates/s, cells, steps, threads, seconds)."""
    threads = threads or os.cpu_count() or 1
    w, s = oracle_solver(args, threads)
    s.solve(1)  # warm-up step
    t0 = time.perf_counter()
    s.solve(1)  # sizes the sample
    one = time.perf_counter() - t0
    n = max(1, min(int(steps_budget_s / max(one, 1e-6)), 50))
    if max_steps is not None:
        n = max(1, min(n, max_steps))
    t0 = time.perf_counter()
    s.solve(n)
    el = time.perf_counter() - t0
    t = s.tables()
    sub = t["subface_cells"]
    return {"value": s.first_ghost * n / el, "cells": int(s.first_ghost), "ghosts": int(s.ncells - s.first_ghost),
            "subface_groups": int(0 if sub is None else sub.shape[1]), "steps": n, "threads": threads,
            "seconds": el}


def parity_record(args, steps=5):
    """The checker of the timed path: the oracle and the library's FP64 and
    mixed paths stepped from the oracle's hom3-numbered tables and initial
    state through the C ABI (the drop-in path), compared after one step and
    after `steps` steps."""
    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200.solver import euler_neumann

    w, o = oracle_solver(args, os.cpu_count() or 1)
    t = o.tables()
    fg = o.first_ghost

    def gpu(prec):
        g = hb.Solver(3, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, prec, cfl=args.cfl, time_end=1e30)
        g.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg,
                   [euler_neumann() for _ in range(6)], t["subface_cells"])
        g.set_state(o.state(0), 0)
        g.reset_time()
        return g

    def max_rel(a, b):
        big = np.abs(b).max()
        return float(max(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-6 * big) for v in range(b.shape[0])))

    def l2_rel(a, b):
        return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))

    g64, gmx = gpu(F.FP64), gpu(F.MIXED)
    out = {"cells": int(fg), "steps": steps}
    for g in (g64, gmx):
        g.solve(1)
    o.solve(1)
    qo = o.state(0)[:, :fg]
    out["fp64_max_rel_after_1"] = max_rel(g64.state(0)[:, :fg], qo)
    out["dt_rel_after_1"] = abs(g64.dt() - o.dt()) / o.dt()
    for g in (g64, gmx):
        g.solve(steps - 1)
    o.solve(steps - 1)
    qo = o.state(0)[:, :fg]
    q64, qmx = g64.state(0)[:, :fg], gmx.state(0)[:, :fg]
    out[f"fp64_max_rel_after_{steps}"] = max_rel(q64, qo)
    out[f"fp64_l2_rel_after_{steps}"] = l2_rel(q64, qo)
    out[f"mixed_l2_rel_after_{steps}"] = l2_rel(qmx, qo)
    out[f"mixed_max_rel_after_{steps}"] = max_rel(qmx, qo)
    out["stage_kernel"] = g64.kernel_info()["kernel"]
    out["what"] = ("oracle (CPU restatement of hom3) vs the library through h3c_set_grid/h3c_set_state with the "
                   "oracle's tables and state; max_rel: max over variables of max|a-b| / max|b|; l2_rel: "
                   "||a-b||_2 / ||b||_2 over all variables")
    return out


def run_reference(args, ws, rank):
    if rank != 0:
        return
    r = cpu_oracle_run(args, steps_budget_s=20.0, max_steps=max(args.steps, 1))
    w_cfg = workload_config(args, {"first_ghost": r["cells"], "ncells": r["cells"] + r["ghosts"],
                                   "subface_groups": r["subface_groups"]})
    ups, n = r["value"], r["steps"]
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": ups, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / n, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": w_cfg,
        "cpu_baseline": {"value": ups, "unit": "cell-updates/s", "cores": r["threads"], "kind": "port",
                         "sample": f"{n} full RK2 steps of the same {r['cells']}-cell grid, timed after two untimed "
                                   "steps (one warm-up, one that sizes the sample to about 20 s); hom3 itself is "
                                   "uncompilable here (Eigen/Boost/MPI absent), so the reference is the oracle's "
                                   "C++ restatement of hom3, OpenMP over all host threads"},
        "e2e": {"value": ups, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args, t):
    cfg = {"workload": "3D Euler hierarchical tree: 64^3 base on [0,1]^3 +2 levels in sphere r=0.25, "
                       "perturbed 3D Riemann (16 Fourier modes, seed 0), outflow BCs, AUSM, RK2"
                       if (args.base_level, args.extra_levels) == (6, 2) else
                       f"3D Euler hierarchical tree: base level {args.base_level} +{args.extra_levels} levels",
           "time_integration": "rk2", "flux": "ausm", "precision": args.precision, "cfl": args.cfl,
           "parallelism": f"replicas x{args.gpus}"}
    if t is not None:
        fg = t["first_ghost"]
        cfg["leaf_cells"] = int(fg)
        cfg["ghost_cells"] = int(t["ncells"] - fg)
        if "subface_groups" in t:
            cfg["subface_groups"] = int(t["subface_groups"])
        else:
            cfg["subface_groups"] = int(0 if t["subface_cells"] is None else t["subface_cells"].shape[1])
    return cfg


def ensemble_measure(args, ws, local, steps, warmup):
    """The batched workload: args.members independent 2D isentropic-vortex
    grids of uneven size (nx, ny in U{32..512}, +1-level patches on 0-30% of
    each box), one launch per stage over all of them (launch shape from the
    autotuner), mixed and FP64; the plain FP64 path one grid at a time; the
    L2 error of the batched runs against the single-instance FP64 runs.
    Returns a dict (the record the bench line carries)."""
    import concurrent.futures as cf

    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import workloads as W
    from hom3_b200.solver import euler_neumann

    from hom3_b200 import shard

    torch.cuda.set_device(local)
    all_ms = W.ensemble_members(args.members)
    # N ranks split the independent instances (no collective on the data path)
    rank = int(os.environ.get("RANK", "0"))
    assign = shard.partition([m["nx"] * m["ny"] for m in all_ms], ws)
    ms = [all_ms[i] for i in assign[rank]]
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:  # the builder releases the GIL
        tables = list(ex.map(W.ensemble_member_tables, ms))

    def ic(mt):
        m, t = mt
        fg = t["first_ghost"]
        q = np.zeros((4, t["ncells"]))
        q[:, :fg] = hb.cell_average(W.vortex_ic(m["beta"], *m["centre"]), t["x_center"][:, :fg], t["length"][:fg], 2)
        return q

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        states = list(ex.map(ic, zip(ms, tables)))
    q0 = np.concatenate(states, axis=1)
    local_cells = sum(t["first_ghost"] for t in tables)
    cells = int(allreduce_sum([local_cells], ws)[0])  # all ranks' instances
    results = {}
    for prec_name in ("mixed", "fp64"):
        prec = F.MIXED if prec_name == "mixed" else F.FP64
        b = hb.Batch(2, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, prec, cfl=args.cfl, time_end=1e30)
        b.set_grids(tables, [[euler_neumann() for _ in range(4)] for _ in tables])
        b.set_state(q0, 0)
        b.reset_time()
        choice, _ = b.autotune(10)
        stream = torch.cuda.ExternalStream(b.stream())
        b.solve(warmup)
        torch.cuda.synchronize()
        barrier(ws)
        l0 = b.launches()
        with ClockSampler(local) as clk:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            b.solve(steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        ms_ = allreduce_max(ev0.elapsed_time(ev1), ws)
        results[prec_name] = dict(value=cells * steps / (ms_ * 1e-3), ms=ms_, choice=choice,
                                  launches=b.launches() - l0, clocks=clk.summary(), state=b.state(0),
                                  kernel=b.kernel_info(), inst=b.instances())
        del b
    # the plain FP64 path without batching: one solver per grid, stepped one after another
    seq = []
    for t, q in zip(tables, states):
        s1 = hb.Solver(2, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, F.FP64, cfl=args.cfl, time_end=1e30)
        s1.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], t["first_ghost"],
                    [euler_neumann() for _ in range(4)], t["subface_cells"])
        s1.set_state(q, 0)
        s1.reset_time()
        s1.solve(warmup)
        seq.append(s1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s1 in seq:  # each grid finishes before the next starts (dt read-back synchronises)
        s1.solve(steps)
        s1.dt()
    torch.cuda.synchronize()
    seq_s = allreduce_max(time.perf_counter() - t0, ws)
    seq_value = cells * steps / seq_s
    # accuracy after the same warmup + steps: batched mixed and batched FP64
    # against the single-instance FP64 runs (relative L2 over all instances)
    single = np.concatenate([s1.state(0) for s1 in seq], axis=1)
    del seq
    qa, qb = results["mixed"].pop("state"), results["fp64"].pop("state")
    results["fp64_inst"] = results["fp64"].pop("inst")
    results["mixed"].pop("inst")
    num_m, num_f, den = allreduce_sum([((qa - single) ** 2).sum(), ((qb - single) ** 2).sum(), (single ** 2).sum()], ws)
    l2_mixed = float(np.sqrt(num_m / den))
    l2_fp64 = float(np.sqrt(num_f / den))
    # per-instance time steps of every rank, gathered in instance order
    dts = shard.gather(list(zip(*results["fp64_inst"][:2])), assign, rank)
    peak, peak_kind = peaks()
    r = results["mixed"]
    bytes_cell_step = 2 * 4 * 8 + 3 * 4 * 8 + 2 * (4 * 4 + 1)  # RK2, 2D: states, int32 neighbours, level byte
    ach = local_cells * bytes_cell_step / (r["ms"] / steps * 1e-3) / 1e9  # this rank's GPU
    return {
        "members": args.members, "leaf_cells": int(cells), "steps": steps, "warmup": warmup,
        "ranks": ws, "instances_per_rank": [len(a) for a in assign],
        "instance_dt_range": [float(min(d for d, _ in dts)), float(max(d for d, _ in dts))],
        "batched_mixed_value": r["value"], "batched_fp64_value": results["fp64"]["value"],
        "plain_fp64_one_grid_at_a_time_value": seq_value,
        "mixed_over_fp64_batched": r["value"] / results["fp64"]["value"],
        "batched_fp64_over_one_at_a_time": results["fp64"]["value"] / seq_value,
        "batched_mixed_over_plain_fp64": r["value"] / seq_value,
        "l2_rel_batched_mixed_vs_single_fp64": l2_mixed, "l2_rel_batched_fp64_vs_single_fp64": l2_fp64,
        "autotune_choice": {"mixed": r["choice"], "fp64": results["fp64"]["choice"]},
        "stage_kernel": {"mixed": r["kernel"], "fp64": results["fp64"]["kernel"]},
        "gpu_launches_mixed": int(r["launches"]), "clocks": r["clocks"],
        "roofline": {"bound": "hbm", "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "achieved": ach,
                     "frac": ach / peak, "what": "whole batched mixed step, algorithmic bytes "
                                                 f"{bytes_cell_step} B per cell-update"},
        "what": "batched: one launch per stage over all instances (autotuned launch shape); plain: one solver "
                "per grid stepped to completion one after another (dt read-back between grids)",
    }


def run_ensemble(args, ws, rank, local):
    """The batched workload alone, as the bench line (see ensemble_measure)."""
    e = ensemble_measure(args, ws, local, args.steps, args.warmup)
    line = {
        "metric": "cell-updates/s", "value": e["batched_mixed_value"], "unit": "cell-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": e["leaf_cells"] / e["batched_mixed_value"] * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32-flux/f64-state",
        "data": "synthetic",
        "config": {"workload": f"{args.members} independent 2D isentropic vortices (nx, ny in U{{32..512}}, "
                               "+1-level patches on 0-30% of each box, beta in U[1,5]), Neumann outflow, AUSM, RK2, "
                               "one launch per stage over all instances of a rank",
                   "leaf_cells": e["leaf_cells"],
                   "parallelism": f"instances split over {ws} rank(s), no collective on the data path"},
        "gpu_launches": e["gpu_launches_mixed"], "clocks": e["clocks"], "roofline": e["roofline"], "batched": e,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_tgv(args, ws, rank, local):
    """3D compressible Navier-Stokes Taylor-Green vortex (periodic [0, 2pi]^3,
    Re 1600, Mach 0.1, Pr 0.71) on a uniform grid, FP64 and mixed precision;
    kinetic-energy dissipation rate of the mixed path against the FP64 path."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200.solver import Condition

    torch.cuda.set_device(local)
    spec = hb.GridSpec(3, [0.0] * 3, [2 * math.pi] * 3, args.tgv_level)
    t = hb.build_tables(spec, spec.cube_boundaries())
    partners = hb.periodic_partners(t, spec)
    fg = t["first_ghost"]
    U, r0, p0 = 0.1, 1.0, 1 / 1.4

    def ic(x):
        u = U * np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
        v = -U * np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
        p = p0 + r0 * U * U / 16.0 * (np.cos(2 * x[0]) + np.cos(2 * x[1])) * (np.cos(2 * x[2]) + 2.0)
        rho = r0 * p / p0
        q = np.zeros((5, x.shape[1]))
        q[0], q[1], q[3] = rho * u, rho * v, rho
        q[4] = p / 0.4 + 0.5 * rho * (u * u + v * v)
        return q

    q0 = np.zeros((5, t["ncells"]))
    q0[:, :fg] = hb.cell_average(ic, t["x_center"][:, :fg], t["length"][:fg], 3)
    out = {}
    for name, prec in (("fp64", F.FP64), ("mixed", F.MIXED)):
        s = hb.Solver(3, F.CNS, F.FLUX_AUSM, F.RUNGE_KUTTA_2, prec, cfl=0.5, cfl_viscous=0.4, Minfty=0.1,
                      ReInfty=1600.0, Pr0=0.71, time_end=1e30)
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg,
                   [Condition(F.BC_PERIODIC) for _ in range(6)])
        s.set_periodic(partners)
        if args.halo_kernel is not None:
            s.set_option(F.OPT_HALO_KERNEL, args.halo_kernel)
        s.set_state(q0, 0)
        s.reset_time()
        stream = torch.cuda.ExternalStream(s.stream())
        s.solve(args.warmup)
        torch.cuda.synchronize()
        ke0 = None
        with ClockSampler(local) as clk:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            s.solve(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        ms = allreduce_max(ev0.elapsed_time(ev1), ws)
        q = s.state(0)[:, :fg]
        ke = 0.5 * ((q[0] ** 2 + q[1] ** 2 + q[2] ** 2) / q[3]).mean()
        # per-kernel device time of further steps, every launch bracketed by events
        s.profile(True)
        s.solve(min(args.steps, 20))
        torch.cuda.synchronize()
        s.profile(False)
        kern = s.profile_read()
        out[name] = dict(value=fg * args.steps * ws / (ms * 1e-3), ms=ms, ke=float(ke), time=s.time(),
                         clocks=clk.summary(), kernels=kern, stage_kernel=s.kernel_info())
    ke_init = float((0.5 * (q0[0, :fg] ** 2 + q0[1, :fg] ** 2) / q0[3, :fg]).mean())
    line = {"metric": "cell-updates/s", "value": out["fp64"]["value"], "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["fp64"]["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"3D CNS Taylor-Green vortex, periodic [0,2pi]^3, uniform {2 ** args.tgv_level}^3, "
                                   "Re 1600, Mach 0.1, Pr 0.71, AUSM + three-point viscous, RK2", "leaf_cells": int(fg)},
            "mixed_value": out["mixed"]["value"], "mixed_over_fp64": out["mixed"]["value"] / out["fp64"]["value"],
            "ke_fp64": out["fp64"]["ke"], "ke_mixed": out["mixed"]["ke"], "ke_initial": ke_init,
            "ke_rel_diff": abs(out["mixed"]["ke"] - out["fp64"]["ke"]) / out["fp64"]["ke"],
            "sim_time": out["fp64"]["time"], "clocks": out["fp64"]["clocks"],
            "stage_kernel": out["fp64"]["stage_kernel"],
            "kernels_ms": {n: {k: {"total_ms": v[0], "launches": v[1]} for k, v in out[n]["kernels"].items()}
                           for n in out}}
    # roofline of the second RK stage: reads lhs and rhs, writes lhs (3 x 5 x 8 B per cell; uniform grid,
    # no table bytes counted); the CNS stage is FP64-arithmetic heavy, so HBM is a lower bound on its time
    peak, peak_kind = peaks()
    st2_ms, st2_n = out["fp64"]["kernels"].get("stage2", (0.0, 0))
    if st2_n:
        ach = fg * 3 * 5 * 8 / (st2_ms / st2_n * 1e-3) / 1e9
        line["roofline"] = {"bound": "hbm", "kernel": "CNS stage (second RK stage)", "achieved": ach, "peak": peak,
                            "unit": "GB/s", "frac": ach / peak, "peak_source": peak_kind,
                            "algorithmic_bytes_per_launch": fg * 3 * 5 * 8, "avg_launch_ms": st2_ms / st2_n,
                            "step_frac": fg * 200 / (out["fp64"]["ms"] / args.steps * 1e-3) / 1e9 / peak}
    if args.tgv_end > 0 and ws == 1:
        line["long_run"] = tgv_long_record(args)
    if rank == 0:
        print(json.dumps(line), flush=True)


def tgv_long_record(args):
    """The Taylor-Green vortex as its configuration specifies it: the oracle's
    tree, conditions and cell-averaged initial state handed to the library
    through the C ABI (FP64 and mixed), the kinetic-energy dissipation rate
    -dKE/dt of the first `tgv_oracle_steps` steps against the FP64 oracle,
    then both GPU paths to `tgv_end` convective time units (t U / L with
    U = 0.1, L = 1: 10 units = 100 time units) with KE sampled along the way."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200.solver import Condition
    from oracle import h3o

    h3o.set_num_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    w = h3o.World(3, [0, 0, 0], [2 * math.pi] * 3, level=args.tgv_level)
    bcs = [h3o.bc(h3o.BC_PERIODIC, g) for g in w.cube_boundaries()]
    o = w.add_solver(h3o.CNS, h3o.AUSM, h3o.RK2, bcs=bcs, ic_kind=h3o.IC_TAYLOR_GREEN, ic=[0.1, 1.0, 1 / 1.4],
                     Minfty=0.1, ReInfty=1600.0, Pr0=0.71, cfl=0.5, cfl_viscous=0.4, time_end=1e30, gamma=1.4,
                     Rspecific=287.058, T0=273.15, rho0=1.225, Sutherland0=110.4)
    o.initialize()
    setup_s = time.perf_counter() - t0
    info, tab = o.info(), o.tables()
    fg = o.first_ghost
    props = {k: info[k] for k in ("cfl", "cfl_viscous", "gamma", "Rspecific", "T0", "rho0", "Minfty", "ReInfty",
                                  "Pr0", "Sutherland0", "time_end")}

    def gpu(prec):
        g = hb.Solver(3, info["physics"], info["flux"], info["ti"], prec, **props)
        g.set_grid(tab["neighbors"], tab["x_center"], tab["length"], tab["bc_idx"], fg,
                   [Condition(k, v) for k, v in info["bcs"]], tab["subface_cells"])
        g.set_periodic(o.partner_cells())
        g.set_state(o.state(0), 0)
        g.reset_time()
        return g

    def ke(q):
        q = q[:, :fg]
        return float((0.5 * (q[0] ** 2 + q[1] ** 2 + q[2] ** 2) / q[3]).mean())

    g64, gmx = gpu(F.FP64), gpu(F.MIXED)
    # ---- the first steps against the oracle ----
    k = args.tgv_oracle_steps
    series = {"oracle": [(0.0, ke(o.state(0)))], "fp64": [(0.0, ke(g64.state(0)))], "mixed": [(0.0, ke(gmx.state(0)))]}
    t1 = time.perf_counter()
    for _ in range(k):
        o.solve(1)
        series["oracle"].append((o.time(), ke(o.state(0))))
    oracle_s = time.perf_counter() - t1
    for name, g in (("fp64", g64), ("mixed", gmx)):
        for _ in range(k):
            g.solve(1)
            series[name].append((g.time(), ke(g.state(0))))

    def rates(ser):
        return [-(b[1] - a[1]) / (b[0] - a[0]) for a, b in zip(ser[:-1], ser[1:])]

    eps = {n: rates(v) for n, v in series.items()}
    rec = {"cells": int(fg), "oracle_steps": k, "oracle_setup_s": setup_s, "oracle_s": oracle_s,
           "oracle_threads": os.cpu_count() or 1}
    if k > 0:
        scale = max(abs(e) for e in eps["oracle"])
        rec["eps_oracle"] = eps["oracle"]
        rec["eps_rel_diff_fp64_vs_oracle"] = max(abs(a - b) for a, b in zip(eps["fp64"], eps["oracle"])) / scale
        rec["eps_rel_diff_mixed_vs_oracle"] = max(abs(a - b) for a, b in zip(eps["mixed"], eps["oracle"])) / scale
        qo = o.state(0)[:, :fg]
        rec["state_max_rel_fp64_vs_oracle"] = float(np.abs(g64.state(0)[:, :fg] - qo).max() / np.abs(qo).max())
        rec["state_l2_rel_mixed_vs_oracle"] = float(np.sqrt(((gmx.state(0)[:, :fg] - qo) ** 2).sum() / (qo ** 2).sum()))
    del o, w
    # ---- both GPU paths on to the end time, KE sampled every `every` steps ----
    t_end = args.tgv_end / 0.1
    every = 50
    for name, g in (("fp64", g64), ("mixed", gmx)):
        ser = [series[name][-1]]
        stream = torch.cuda.ExternalStream(g.stream())
        steps, dev_ms = 0, 0.0
        while g.time() < t_end:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            g.solve(every)
            ev1.record(stream)
            torch.cuda.synchronize()
            dev_ms += ev0.elapsed_time(ev1)
            steps += every
            ser.append((g.time(), ke(g.state(0))))
        e = rates(ser)
        i = int(np.argmax(e)) if e else 0
        rec[name] = {"steps": steps + k, "time": g.time(), "convective_time": g.time() * 0.1,
                     "device_ms": dev_ms, "value": fg * steps / (dev_ms * 1e-3) if dev_ms else None,
                     "ke_end": ser[-1][1], "ke_start": series[name][0][1],
                     "eps_peak": e[i] if e else None,
                     "eps_peak_convective_time": 0.5 * (ser[i][0] + ser[i + 1][0]) * 0.1 if e else None,
                     "samples": [(round(a * 0.1, 4), b) for a, b in ser[:: max(1, len(ser) // 40)]]}
        series[name + "_long"] = ser
    a, b = rates(series["fp64_long"]), rates(series["mixed_long"])
    m = min(len(a), len(b))
    if m:
        rec["eps_rel_diff_mixed_vs_fp64"] = max(abs(x - y) for x, y in zip(a[:m], b[:m])) / max(abs(x) for x in a[:m])
    rec["what"] = ("KE = mean of rho |u|^2 / 2 over the cells; eps = -dKE/dt between samples (every step against "
                   "the oracle, every 50 steps to the end); tables and initial state are the oracle's")
    return rec


def run_decomposed(args, ws, rank, local):
    """The default workload's one grid split over the ranks (hom3_b200/domain.py):
    each rank steps one Morton-range subdomain; before every stage the ranks
    exchange the cells their faces read (NCCL send/recv of device buffers),
    and before every step they take the minimum time step (NCCL all-reduce).
    Strong scaling: the total work is the one grid whatever N.  Device time
    with CUDA events on each rank's stream, max over ranks."""
    import torch
    import torch.distributed as dist

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import domain
    from hom3_b200 import workloads as W

    torch.cuda.set_device(local)
    spec = W.riemann3d_spec(args.base_level, args.extra_levels)
    t = hb.build_tables(spec, spec.cube_boundaries())
    fg = t["first_ghost"]
    q = np.zeros((5, t["ncells"]))
    q[:, :fg] = hb.cell_average(W.riemann3d_ic(W.fourier_modes()), t["x_center"][:, :fg], t["length"][:fg], 3)
    prec = F.MIXED if args.precision == "mixed" else F.FP64

    def make():
        return hb.Solver(3, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, prec, cfl=args.cfl, time_end=1e30)

    group = dist.group.WORLD if ws > 1 else None
    if ws == 1:  # one rank: a process group of one, so the same exchange code runs
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        dist.init_process_group("gloo", rank=0, world_size=1)
    d = domain.DomainSolver(t, 3, make, W.riemann3d_conditions(), rank, ws, group)
    d.set_state(q)
    stream = torch.cuda.ExternalStream(d.s.stream())
    d.solve(args.warmup)
    torch.cuda.synchronize()
    barrier(ws)
    with ClockSampler(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        d.solve(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = allreduce_max(ev0.elapsed_time(ev1), ws)
    halo = d.sub.halo.size
    line = {"metric": "cell-updates/s", "value": fg * args.steps / (ms * 1e-3), "unit": "cell-updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if prec == F.FP64 else "f32-flux/f64-state", "data": "synthetic",
            "config": dict(workload_config(args, t), parallelism=f"domain decomposition x{ws}"),
            "cells_per_rank": int(d.sub.cells.size), "exchange_ghosts_rank0": int(halo),
            "clocks": clk.summary(),
            "what": "one grid split along the Morton order; per stage an exchange of the cells each "
                    "subdomain's faces read, per step an all-reduce of the minimum time step"}
    if ws == 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_vortex(args, ws, rank, local):
    """2D Euler isentropic vortex on a uniform 256^2 grid over [0, 10]^2,
    periodic, beta 5, centre (5, 5), free stream rho = u = v = p = 1, CFL 0.5:
    the second-order scheme (LSQ gradients + MUSCL + Venkatakrishnan limiter,
    SSP-RK3) in FP64 and mixed precision, and hom3's first-order AUSM/RK2 for
    comparison.  Each result's density L2 error against the exact solution
    (the initial vortex advected by (t, t)) is reported beside its speed."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import workloads as W
    from hom3_b200.solver import Condition

    torch.cuda.set_device(local)
    level = args.vortex_level
    spec = hb.GridSpec(2, [0.0, 0.0], [10.0, 10.0], level)
    t = hb.build_tables(spec, spec.cube_boundaries())
    partners = hb.periodic_partners(t, spec)
    fg = t["first_ghost"]
    f0 = W.vortex_ic(5.0, 5.0, 5.0)
    q0 = np.zeros((4, t["ncells"]))
    q0[:, :fg] = hb.cell_average(f0, t["x_center"][:, :fg], t["length"][:fg], 2)

    def exact(time_):
        def f(x):
            return f0(np.mod(x - time_, 10.0))
        return hb.cell_average(f, t["x_center"][:, :fg], t["length"][:fg], 2)

    runs = (("muscl_rk3_fp64", F.SSPRK3, F.RECON_MUSCL, F.FP64), ("muscl_rk3_mixed", F.SSPRK3, F.RECON_MUSCL, F.MIXED),
            ("first_order_rk2_fp64", F.RUNGE_KUTTA_2, F.RECON_NONE, F.FP64))
    out = {}
    for name, ti, rec, prec in runs:
        s = hb.Solver(2, F.EULER, F.FLUX_AUSM, ti, prec, reconstruction=rec, limiter_k=1.0, cfl=0.5,
                      time_end=1e30)
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg,
                   [Condition(F.BC_PERIODIC) for _ in range(4)])
        s.set_periodic(partners)
        stream = torch.cuda.ExternalStream(s.stream())
        s.set_state(q0, 0)
        s.reset_time()
        s.solve(args.warmup)  # warm-up (graph capture), then the timed run from the initial state
        s.set_state(q0, 0)
        s.reset_time()
        torch.cuda.synchronize()
        l0 = s.launches()
        with ClockSampler(local) as clk:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            s.solve(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        ms = allreduce_max(ev0.elapsed_time(ev1), ws)
        launches = s.launches() - l0
        q = s.state(0)[:, :fg]
        tt = s.time()
        ex = exact(tt)
        s.profile(True)
        s.solve(min(args.steps, 50))
        torch.cuda.synchronize()
        s.profile(False)
        kern = s.profile_read()
        out[name] = dict(value=fg * args.steps * ws / (ms * 1e-3), ms=ms, time=tt, launches=int(launches),
                         l2_rho=float(np.sqrt(((q[2] - ex[2]) ** 2).mean())), q=q, clocks=clk.summary(),
                         kernels_ms={k: {"total_ms": v[0], "launches": v[1]} for k, v in kern.items()})
    d = out["muscl_rk3_mixed"]["q"] - out["muscl_rk3_fp64"]["q"]
    l2_mixed_vs_fp64 = float(np.sqrt((d ** 2).mean() / (out["muscl_rk3_fp64"]["q"] ** 2).mean()))
    a = out["muscl_rk3_fp64"]
    line = {"metric": "cell-updates/s", "value": a["value"], "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": a["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"2D Euler isentropic vortex, uniform {2 ** level}^2 on [0,10]^2, periodic, "
                                   "beta 5, centre (5,5), LSQ gradients + MUSCL + Venkatakrishnan (K 1), "
                                   "SSP-RK3, CFL 0.5", "leaf_cells": int(fg),
                       "l2": "working set (3 states + gradients) is L2-resident; no flush"},
            "gpu_launches": a["launches"], "sim_time": a["time"], "l2_rho_error": a["l2_rho"],
            "runs": {k: {kk: vv for kk, vv in v.items() if kk != "q"} for k, v in out.items()},
            "mixed_over_fp64": out["muscl_rk3_mixed"]["value"] / a["value"],
            "mixed_vs_fp64_rel_l2": l2_mixed_vs_fp64, "clocks": a["clocks"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_advection(args, ws, rank, local):
    """hom3's advection test (advection_fv_solver_test.cpp:51-125) at a larger
    size: the disc q = 1 (r = 0.08 around (0.25, 0.5)) in q = 0.1 carried by
    the test's rotating velocity field on a uniform 2^L x 2^L grid over [0,1]^2,
    characteristic conditions, forward Euler.  The timed run uses the LLF flux
    at CFL 0.5; hom3's own upwind flux at CFL 1 (unstable where the face
    velocity is negative: it negates u_L q_L) is timed beside it."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import workloads as W
    from hom3_b200.solver import adv_characteristic

    torch.cuda.set_device(local)
    level = args.adv_level
    spec = hb.GridSpec(2, [0.0, 0.0], [1.0, 1.0], level)
    t = hb.build_tables(spec, spec.cube_boundaries(), device=True)
    fg, n = t["first_ghost"], t["ncells"]
    u = W.rotation_velocity(t["x_center"])
    q0 = np.zeros((1, n))
    q0[:, :fg] = hb.cell_average(W.disc_ic(), t["x_center"][:, :fg], t["length"][:fg], 2)
    out = {}
    for name, flux, cfl in (("llf_fe", F.FLUX_LLF, 0.5), ("hom3_upwind_fe", F.FLUX_UPWIND, 1.0)):
        s = hb.Solver(2, F.ADVECTION, flux, F.EULER_FORWARD, F.FP64, cfl=cfl, time_end=1e30)
        s.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg, [adv_characteristic()] * 4)
        s.set_velocity(u)
        stream = torch.cuda.ExternalStream(s.stream())
        s.set_state(q0, 0)
        s.reset_time()
        s.solve(args.warmup)
        s.set_state(q0, 0)
        s.reset_time()
        torch.cuda.synchronize()
        l0 = s.launches()
        with ClockSampler(local) as clk:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            s.solve(args.steps)
            ev1.record(stream)
            torch.cuda.synchronize()
        ms = allreduce_max(ev0.elapsed_time(ev1), ws)
        launches = s.launches() - l0
        q = s.state(0)[0, :fg]
        s.profile(True)
        s.solve(min(args.steps, 50))
        torch.cuda.synchronize()
        s.profile(False)
        kern = s.profile_read()
        out[name] = dict(value=fg * args.steps * ws / (ms * 1e-3), ms=ms, launches=int(launches),
                         q_min=float(q.min()), q_max=float(q.max()), clocks=clk.summary(),
                         kernels_ms={k: {"total_ms": v[0], "launches": v[1]} for k, v in kern.items()})
    a = out["llf_fe"]
    st = a["kernels_ms"].get("stage1", {"total_ms": 0.0, "launches": 0})
    stage_ms = st["total_ms"] / max(st["launches"], 1)
    # algorithmic bytes per cell and stage: q read + written (16 B), the cell's velocity (16 B),
    # 4 int32 neighbours (16 B) and the level byte
    b_cell = 8 + 8 + 16 + 16 + 1
    peak, peak_src = peaks()
    achieved = fg * b_cell / (stage_ms * 1e-3) / 1e9 if stage_ms > 0 else None
    line = {"metric": "cell-updates/s", "value": a["value"], "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": a["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"2D advection (hom3's rotating-disc test) on a uniform {2 ** level}^2 grid, "
                                   "characteristic conditions, LLF flux, forward Euler, CFL 0.5",
                       "leaf_cells": int(fg), "l2": "working set (state, velocity, tables) exceeds the 126 MB L2"},
            "roofline": {"bound": "hbm", "kernel": "k_stage (advection)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                         "algorithmic_bytes_per_cell": b_cell, "avg_launch_ms": stage_ms, "peak_source": peak_src},
            "gpu_launches": a["launches"], "runs": out, "clocks": a["clocks"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_cht(args, ws, rank, local):
    """Conjugate heat transfer: CNS channel 512 x 128 over a heat-conducting
    solid 512 x 64 in one level-9 root cell, conductivity ratio 10, solid
    initial temperature 1 + 0.1 (smooth 16-mode field, seed 1); each step
    coupling::apply (common dt, Tr0 = 0.01), one CNS step, one heat step
    (coupled_cns_heat_test.cpp:235-248).  Unit: one cell (fluid or solid)
    advanced one step."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import workloads as W

    torch.cuda.set_device(local)
    d = W.cht_setup()
    tf, ts = d["tables_fluid"], d["tables_solid"]
    fgf, fgs = tf["first_ghost"], ts["first_ghost"]

    def make():
        cns = hb.Solver(2, F.CNS, F.FLUX_AUSM, F.EULER_FORWARD, F.FP64, time_end=1e30, **d["props"])
        heat = hb.Solver(2, F.HEAT, F.FLUX_AUSM, F.EULER_FORWARD, F.FP64, cfl=0.5, time_end=1e30)
        cns.set_grid(tf["neighbors"], tf["x_center"], tf["length"], tf["bc_idx"], fgf, d["conditions_fluid"])
        heat.set_grid(ts["neighbors"], ts["x_center"], ts["length"], ts["bc_idx"], fgs, d["conditions_solid"])
        cns.set_partner(heat, d["partners_fluid"])
        heat.set_partner(cns, d["partners_solid"])
        cns.set_state(d["q_fluid"], 0)
        heat.set_state(d["q_solid"], 0)
        cns.reset_time()
        heat.reset_time()
        return cns, heat

    cns, heat = make()
    stream = torch.cuda.ExternalStream(cns.stream())
    Tr0 = 0.01

    def steps(n):
        hb.cht_solve(Tr0, cns, heat, n)

    steps(args.warmup)
    torch.cuda.synchronize()
    l0 = cns.launches() + heat.launches()
    with ClockSampler(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        steps(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = allreduce_max(ev0.elapsed_time(ev1), ws)
    launches = cns.launches() + heat.launches() - l0
    # the same steps one call per solver and step (hom3's loop shape), for comparison
    c2, h2 = make()
    for _ in range(args.warmup):
        hb.couple_cht(Tr0, c2, h2)
        c2.solve(1)
        h2.solve(1)
    torch.cuda.synchronize()
    s2 = torch.cuda.ExternalStream(c2.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s2)
    for _ in range(args.steps):
        hb.couple_cht(Tr0, c2, h2)
        c2.solve(1)
        h2.solve(1)
    e1.record(s2)
    torch.cuda.synchronize()
    ms_loop = e0.elapsed_time(e1)
    Ts = heat.state(0)[0, :fgs]
    cells = fgf + fgs
    adj = cht_adjoint_measure(args, d, make, Tr0) if args.adjoint_steps > 0 else None
    line = {"metric": "cell-updates/s", "value": cells * args.steps * ws / (ms * 1e-3), "unit": "cell-updates/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "2D conjugate heat transfer: CNS 512x128 over heat 512x64 in one level-9 root "
                                   "cell, conductivity ratio 10, Minfty 0.2, ReInfty 100, Tr0 0.01, forward Euler, "
                                   "solid T0 = T_inf (1 + 0.1 f), f 16 Fourier modes seed 1",
                       "fluid_cells": int(fgf), "solid_cells": int(fgs)},
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "per_solver_loop_value": cells * args.steps / (ms_loop * 1e-3),
            "solid_T_range": [float(Ts.min()), float(Ts.max())], "time": cns.time()}
    if adj is not None:
        line["adjoint"] = adj
    if rank == 0:
        print(json.dumps(line), flush=True)


def cht_adjoint_measure(args, d, make, Tr0):
    """Adjoint of the total interface heat flux after N coupled steps with
    respect to the solid's initial temperature (checkpoints every 100 steps,
    time steps frozen): time against the forward loop, and central differences
    of the frozen-dt coupled map in a few random solid directions (seed 2).
    J = sum over the solid's interface ghosts of (T_b - T_g) = sum 2 (T_b - T_f) / (1 + kappa)."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    tf, ts = d["tables_fluid"], d["tables_solid"]
    fgf, fgs = tf["first_ghost"], ts["first_ghost"]
    n = min(args.steps, 2000)
    kappa = float(d["conditions_solid"][3].values[0])
    ghosts = np.arange(fgs, ts["ncells"])
    coupled = ts["bc_idx"][fgs:] == 3
    nb = ts["neighbors"][:, fgs:]
    bcell = np.where((nb >= 0) & (nb < fgs), nb, -1).max(axis=0)
    pf = d["partners_solid"]
    c = 2.0 / (1.0 + kappa)

    def objective(cns, heat):
        qf, qs = cns.state(0), heat.state(0)
        rho = qf[2]
        T = 1.4 * 0.4 * (qf[3] - 0.5 * (qf[0] ** 2 + qf[1] ** 2) / rho) / rho
        g = ghosts[coupled] - fgs
        return float((c * (qs[0, bcell[g]] - T[pf[g]])).sum())

    def cotangents(cns):
        qf = cns.state(0)
        lf, ls = np.zeros_like(qf), np.zeros((1, ts["ncells"]))
        g = ghosts[coupled] - fgs
        np.add.at(ls[0], bcell[g], c)
        P = pf[g]
        rho, u, v, E = qf[2, P], qf[0, P] / qf[2, P], qf[1, P] / qf[2, P], qf[3, P]
        p = 0.4 * (E - 0.5 * rho * (u * u + v * v))
        np.add.at(lf[0], P, -c * (-1.4 * 0.4 * u / rho))
        np.add.at(lf[1], P, -c * (-1.4 * 0.4 * v / rho))
        np.add.at(lf[2], P, -c * 1.4 * (0.5 * 0.4 * (u * u + v * v) - p / rho) / rho)
        np.add.at(lf[3], P, -c * 1.4 * 0.4 / rho)
        return lf, ls

    # forward loop time and the final state's cotangents
    cns, heat = make()
    stream = torch.cuda.ExternalStream(cns.stream())  # the coupled pair's shared stream
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    hb.cht_solve(Tr0, cns, heat, n)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    lf, ls = cotangents(cns)
    J0 = objective(cns, heat)
    cns, heat = make()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gf, gs, dts = hb.cht_adjoint(Tr0, cns, heat, n, lf, ls, every=100)
    adj_s = time.perf_counter() - t0
    # the same call again with every launch bracketed by events: where the time goes
    c3, h3 = make()
    c3.profile(True)
    h3.profile(True)
    hb.cht_adjoint(Tr0, c3, h3, n, lf, ls, every=100)
    torch.cuda.synchronize()
    kern = {("fluid " + k): v for k, v in c3.profile_read().items()}
    kern.update({("solid " + k): v for k, v in h3.profile_read().items()})
    # lf, ls: dJ/dq_N, dJ/dT_N at the final states (J is linear in T, nonlinear in the fluid state)
    rng = np.random.default_rng(2)

    def J_of(Ts0):
        c2, h2 = make()
        h2.set_state(Ts0, 0)
        h2.reset_time()
        c2.reset_time()
        for i in range(n):
            c2.solve_dt([dts[0, i]])
            h2.solve_dt([dts[1, i]])
        return objective(c2, h2)

    worst = 0.0
    ndir = 32  # random solid directions (seed 2)
    for _ in range(ndir):
        dT = np.zeros_like(d["q_solid"])
        dT[0, :fgs] = rng.standard_normal(fgs)
        eps = 1e-6
        fd = (J_of(d["q_solid"] + eps * dT) - J_of(d["q_solid"] - eps * dT)) / (2 * eps)
        ad = float((gs * dT).sum())
        worst = max(worst, abs(fd - ad) / max(abs(fd), np.abs(gs * dT).sum() * 1e-3))
    return {"steps": n, "checkpoint_every": 100, "objective": "sum of the interface heat flux at the last step",
            "J": J0, "forward_ms": fwd_ms, "adjoint_ms": adj_s * 1e3, "ratio": adj_s * 1e3 / fwd_ms,
            "fd_directions": ndir, "fd_worst_rel": worst,
            "kernels_ms": {k: {"total_ms": v[0], "launches": v[1]} for k, v in kern.items()},
            "what": "h3c_cht_adjoint (forward with checkpoints, coupled recompute, backward; host arrays) / "
                    "h3c_cht_solve of the same steps"}


def mixed_record(args, t, q0, ws, local, fp64_value):
    """The default workload with FP32 face fluxes and FP64 state, update, dt
    and sums: device-timed cell-updates/s over the same K steps as the FP64
    line, and its ratio to the FP64 value."""
    import torch

    import hom3_b200 as hb
    from hom3_b200 import _ffi as F
    from hom3_b200 import workloads as W

    fg = t["first_ghost"]
    m = hb.Solver(3, F.EULER, F.FLUX_AUSM, F.RUNGE_KUTTA_2, F.MIXED, cfl=args.cfl, time_end=1e30)
    m.set_grid(t["neighbors"], t["x_center"], t["length"], t["bc_idx"], fg, W.riemann3d_conditions(),
               t["subface_cells"])
    m.set_state(q0, 0)
    m.reset_time()
    tune = None
    if args.euler_kernel is not None:
        m.set_option(F.OPT_EULER_KERNEL, args.euler_kernel)
    elif not args.no_autotune:
        choice, _ = m.autotune(10)
        tune = {"choice": choice, "kernel": m.kernel_info()["kernel"]}
    stream = torch.cuda.ExternalStream(m.stream())
    m.solve(args.warmup)
    torch.cuda.synchronize()
    barrier(ws)
    with ClockSampler(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        m.solve(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = allreduce_max(ev0.elapsed_time(ev1), ws)
    v = fg * args.steps * ws / (ms * 1e-3)
    return {"value": v, "unit": "cell-updates/s", "ms_per_step": ms / args.steps, "mixed_over_fp64": v / fp64_value,
            "dtype": "f32-flux/f64-state", "stage_kernel": m.kernel_info()["kernel"], "autotune": tune,
            "clocks": clk.summary(),
            "what": "same tree, state, steps and timing as the FP64 line; FP32 face states and fluxes, FP64 "
                    "state, residual, update and dt"}


def measure_adjoint(s, q0, nsteps, stream, fg):
    """Time h3c_adjoint of J = <lambda, q_N> over nsteps RK2 steps against the
    same nsteps of h3c_solve (CUDA events on the solver's stream, both from the
    same initial state; cotangent and gradient are device arrays)."""
    import torch
    rng = np.random.default_rng(5)
    lam = torch.from_numpy(rng.standard_normal(q0.shape)).cuda()
    grad = torch.empty_like(lam)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    # warm-up: allocates the workspace once
    s.set_state(q0, 0)
    s.reset_time()
    s.adjoint(nsteps, lam, every=0, out=grad)
    s.set_state(q0, 0)
    s.reset_time()
    torch.cuda.synchronize()
    ev[0].record(stream)
    s.solve(nsteps)
    ev[1].record(stream)
    torch.cuda.synchronize()
    s.set_state(q0, 0)
    s.reset_time()
    torch.cuda.synchronize()
    s.profile(True)
    ev[2].record(stream)
    s.adjoint(nsteps, lam, every=0, out=grad)
    ev[3].record(stream)
    torch.cuda.synchronize()
    s.profile(False)
    kern = s.profile_read()
    fwd_ms = ev[0].elapsed_time(ev[1])
    adj_ms = ev[2].elapsed_time(ev[3])
    ak_ms, ak_n = kern.get("adjoint", (0.0, 0))
    # the same adjoint with the per-cell gather in place of the tile kernel
    from hom3_b200 import _ffi as F
    s.set_option(F.OPT_TILE_KERNEL, 0)
    s.set_state(q0, 0)
    s.reset_time()
    torch.cuda.synchronize()
    s.profile(True)
    s.adjoint(nsteps, lam, every=0, out=grad)
    torch.cuda.synchronize()
    s.profile(False)
    gk_ms, gk_n = s.profile_read().get("adjoint", (0.0, 0))
    s.set_option(F.OPT_TILE_KERNEL, 1)
    # algorithmic bytes of one adjoint-stage launch: stage state + cotangent in, cotangent out
    # (+ the extra cotangent of the second launch of a step, counted in the mean) and the tables
    b_launch = fg * (3 * 5 * 8 + 6 * 4 + 1) + 0.5 * fg * 5 * 8
    return {"steps": nsteps, "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "ratio": adj_ms / fwd_ms,
            "what": "h3c_adjoint (forward with checkpoints + backward sweep, device cotangent) / h3c_solve of "
                    "the same steps; the library chose the checkpoint interval",
            "adjoint_kernel_ms": ak_ms / max(ak_n, 1), "adjoint_launches": ak_n,
            "per_cell_gather_kernel_ms": gk_ms / max(gk_n, 1),
            "kernels_ms": {k: round(v[0], 3) for k, v in kern.items()},
            "adjoint_kernel_gbs": b_launch / (ak_ms / max(ak_n, 1) * 1e-3) / 1e9 if ak_n else None,
            "grad_finite": bool(torch.isfinite(grad).all().item())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--base-level", type=int, default=6)
    ap.add_argument("--extra-levels", type=int, default=2)
    ap.add_argument("--cfl", type=float, default=0.4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle comparison of the default workload")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision record of the default workload")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-ensemble record")
    ap.add_argument("--halo-kernel", type=int, default=None,
                    help="1: stage tiles into shared memory (the library's default), 0: the kernels without it")
    ap.add_argument("--decompose", action="store_true",
                    help="split the default workload's one grid over the N ranks (strong scaling) "
                         "instead of running N replicas")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the library's default Euler stage launch instead of h3c_autotune's choice")
    ap.add_argument("--euler-kernel", type=int, default=None,
                    help="Euler stage kernel: 0 halo-staged tile, 1 per-lane tile, 2 per cell, 3 warp-tiled, 4 per-lane tile "
                         "of 512 cells (default: the autotuner's choice)")
    ap.add_argument("--workload", default="riemann3d",
                    choices=["riemann3d", "ensemble", "tgv", "vortex", "cht", "advection"])
    ap.add_argument("--adv-level", type=int, default=11)
    ap.add_argument("--vortex-level", type=int, default=8)
    ap.add_argument("--tgv-level", type=int, default=7)
    ap.add_argument("--tgv-end", type=float, default=0.0,
                    help="TGV: also run from the oracle's state to this convective time (0: timing only)")
    ap.add_argument("--tgv-oracle-steps", type=int, default=3,
                    help="TGV long run: steps compared with the FP64 oracle before the GPU-only run")
    ap.add_argument("--members", type=int, default=256)
    ap.add_argument("--adjoint-steps", type=int, default=50)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_setup()
    if args.workload == "ensemble" and args.impl == "ours":
        run_ensemble(args, ws, rank, local)
        return
    if args.decompose and args.impl == "ours":
        run_decomposed(args, ws, rank, local)
        return
    if args.workload == "tgv" and args.impl == "ours":
        run_tgv(args, ws, rank, local)
        return
    if args.workload == "vortex" and args.impl == "ours":
        run_vortex(args, ws, rank, local)
        return
    if args.workload == "cht" and args.impl == "ours":
        run_cht(args, ws, rank, local)
        return
    if args.workload == "advection" and args.impl == "ours":
        run_advection(args, ws, rank, local)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return

    import torch
    torch.cuda.set_device(local)
    s, t, q0, _ = build_workload(args)
    fg, n = t["first_ghost"], t["ncells"]
    stream = torch.cuda.ExternalStream(s.stream())
    state_bytes = 5 * n * 8
    # ---- device-resident timing ('value') ----
    s.set_state(q0, 0)
    s.reset_time()
    tune = None
    if args.euler_kernel is None and not args.no_autotune:
        # the stage kernel and launch shape for this GPU, timed from the initial state (which it restores)
        choice, tune_ms = s.autotune(10)
        tune = {"choice": choice, "ms_per_step": tune_ms, "kernel": s.kernel_info()["kernel"]}
    with ClockSampler(local) as clk:
        s.solve(args.warmup)
        torch.cuda.synchronize()
        barrier(ws)
        l0 = s.launches()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.solve(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        launches = s.launches() - l0
        # per-kernel durations: the same steps again with every launch bracketed by events
        s.profile(True)
        s.solve(min(args.steps, 100))
        torch.cuda.synchronize()
        s.profile(False)
        kern = s.profile_read()
    barrier(ws)
    ms_max = allreduce_max(ms, ws)
    status = s.status()
    value = fg * args.steps * ws / (ms_max * 1e-3)
    # ---- end-to-end through the C ABI with host buffers ('e2e') ----
    pinned = torch.empty((5, n), dtype=torch.float64, pin_memory=True).numpy()
    pinned[:] = q0
    out = torch.empty((5, n), dtype=torch.float64, pin_memory=True).numpy()
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    s.set_state(pinned, 0)          # H2D of the initial state
    s.reset_time()
    for _ in range(args.steps):     # hom3's run loop: solve, then read dt (utilities.hpp:103-110)
        s.solve(1)
        dt = s.dt()
        if not (1e-300 <= dt <= 1e300):
            raise RuntimeError("solution diverged")
    s.state(0, out=out)             # D2H of the final state
    e2e_s = time.perf_counter() - t0
    e2e_s = allreduce_max(e2e_s, ws)
    e2e = fg * args.steps * ws / e2e_s
    # ---- the mixed-precision path (FP32 face fluxes, FP64 state) on the same tree ----
    mixed = None
    if not args.no_mixed and args.precision == "fp64":
        mixed = mixed_record(args, t, q0, ws, local, value)
    # ---- discrete adjoint: time of h3c_adjoint (its forward included) over the forward alone ----
    adj = None
    if args.adjoint_steps > 0:
        adj = measure_adjoint(s, q0, args.adjoint_steps, stream, fg)
    # ---- roofline of the dominant kernel (second RK stage) ----
    peak, peak_kind = peaks()
    st2_ms, st2_n = kern.get("stage2", (0.0, 0))
    st1_ms, st1_n = kern.get("stage1", (0.0, 0))
    bytes_st2 = fg * (3 * 5 * 8 + 6 * 4 + 1)      # read lhs, rhs; write lhs; int32 neighbours; level byte
    bytes_st1 = fg * (2 * 5 * 8 + 6 * 4 + 1)
    st2_avg = st2_ms / max(st2_n, 1)
    achieved = bytes_st2 / (st2_avg * 1e-3) / 1e9 if st2_n else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "stage2_traffic.json")
    if os.path.exists(tp):
        try:
            d = json.load(open(tp))
            traffic = d["dram_bytes_per_leaf_cell"] * fg
        except Exception:
            traffic = None
    step_bytes = bytes_st1 + bytes_st2
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32-flux/f64-state",
        "data": "synthetic", "config": workload_config(args, t),
        "roofline": {"bound": "hbm", "kernel": "k_stage (second RK stage)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": bytes_st2,
                     "avg_launch_ms": st2_avg,
                     "step_frac": (step_bytes * st2_n / ((st1_ms + st2_ms) * 1e-3) / 1e9 / peak)
                     if st1_n and st2_n and st1_n == st2_n else None},
        "kernels_ms": {k: {"total_ms": v[0], "launches": v[1]} for k, v in kern.items()},
        "kernels_ms_note": "event-bracketed launches of min(K, 100) further steps run right after the timed region",
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "e2e": {"value": e2e, "unit": "cell-updates/s",
                "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": 8 + state_bytes / args.steps,
                "what": "C-ABI run loop with host buffers: h3c_set_state (pinned host) + K x (h3c_solve(1) + "
                        "h3c_dt read-back) + h3c_get_state"},
        "working_set_mb": round((2 * state_bytes + 6 * 4 * n + n) / 2 ** 20, 1),
        "l2": "no flush: the working set (both states + tables) exceeds the 126 MB L2",
        "device_status": status,
    }
    if adj is not None:
        line["adjoint"] = adj
    line["grid_build"] = getattr(args, "grid_build", None)
    line["stage_kernel"] = s.kernel_info()
    line["autotune"] = tune
    r64, r32 = hb_fma_rates()
    line["fma_rates"] = {"fp64_tflops": 2 * r64 / 1e12, "fp32_tflops": 2 * r32 / 1e12,
                         "what": "h3c_fma_rates: register-only FMA chains on this GPU (1 FMA = 2 flops); the FP64 "
                                 "rate bounds the stage kernels' face arithmetic"}
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        r = cpu_oracle_run(args)
        r1 = cpu_oracle_run(args, steps_budget_s=8.0, threads=1)
        line["cpu_baseline"] = {
            "value": r["value"], "unit": "cell-updates/s", "cores": r["threads"], "kind": "port",
            "sample": f"{r['steps']} RK2 steps of the same {r['cells']}-cell workload, {r['seconds']:.1f} s, after "
                      "one warm-up and one sizing step; OpenMP over all host threads",
            "single_thread": {"value": r1["value"], "unit": "cell-updates/s", "cores": 1, "kind": "port",
                              "sample": f"{r1['steps']} RK2 steps, {r1['seconds']:.1f} s (hom3's own execution model "
                                        "is serial)"}}
    if ws == 1 and rank == 0 and not args.no_parity:
        line["parity"] = parity_record(args)
    if mixed is not None:
        if "parity" in line:
            mixed["l2_rel_vs_fp64_oracle"] = line["parity"]["mixed_l2_rel_after_5"]
            mixed["l2_what"] = "after 5 steps from the oracle's state, the parity record's comparison"
        line["mixed"] = mixed
    if not args.no_batched:
        line["batched"] = ensemble_measure(args, ws, local, steps=min(args.steps, 200), warmup=args.warmup)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
