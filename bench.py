"""Benchmark of the B200 solve path (one JSON line on rank 0).

Workload (default ``iccg64``): the plain FP64 ICCG drop-in on a 3-D 7-point
Laplacian, 64^3 interior grid (262,144 unknowns, 1,810,432 nonzeros), RHS
uniform[-1,1] from numpy seed 0, IC shift 1.05, ABMC (block 4, 4 target
colours), tol 1e-10, maxiter 2000. One step = one complete
SparseSolvSolver.Solve (FreeDofs view, ABMC ordering, device IC(0)
factorisation, CG to tolerance) on a fresh solver object with the matrix and
b resident in HBM; metric = time-to-solution (s), lower is better.

``--impl reference`` times the reference's own CPU implementation (its headers
compiled into oracle/_ref/libssv_ref.so, OpenMP over all host cores) on the
same workload. Multi-GPU: independent replicas (one per rank, no collective
on the data path), max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "ngsolve-sparsesolv_b200"))

METRIC = "time-to-solution @1e-10 (s)"
UNIT = "s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _workload(name):
    import numpy as np
    from sparsesolv_ngsolve import problems as P
    if name == "iccg64":
        A = P.laplacian_7pt(64)
        b = P.random_rhs(A.shape[0], 0)
        cfg = dict(method="ICCG", tol=1e-10, maxiter=2000, shift=1.05, use_abmc=True, abmc_block_size=4,
                   abmc_num_colors=4)
        desc = {"workload": "iccg64: ICCG FP64, 3-D 7-point Laplacian 64^3 (262,144 rows, 1,810,432 nnz), "
                            "IC shift 1.05, ABMC block 4 / 4 colours, tol 1e-10",
                "rows": int(A.shape[0]), "nnz": int(A.nnz), "method": "ICCG", "use_abmc": True,
                "tol": 1e-10, "rhs": "uniform[-1,1], numpy default_rng(0)"}
        return A, b, cfg, desc
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(A, b, cfg, budget_s=10.0):
    """The reference CPU path (oracle/_ref, else the oracle port) on host cores."""
    from oracle import oracle as O
    ref = O.reference()
    which = "ref" if ref is not None else "port"
    cores = os.cpu_count() or 1
    if ref is not None:
        ref.ref_set_threads(cores)
    else:
        cores = 1
    c = O.default_config(use_abmc=int(cfg["use_abmc"]), max_iterations=cfg["maxiter"], tolerance=cfg["tol"],
                         shift_parameter=cfg["shift"], abmc_block_size=cfg["abmc_block_size"],
                         abmc_num_colors=cfg["abmc_num_colors"])
    times, iters = [], None
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        _, r, _ = O.solve(A, b, cfg["method"], c, which=which)
        times.append(time.perf_counter() - t0)
        iters = r.iterations
        if time.perf_counter() > t_end or len(times) >= 50:
            break
    return {"value": statistics.mean(times), "unit": UNIT, "cores": cores,
            "kind": "reference" if which == "ref" else "port",
            "sample": f"{len(times)} full solves of the workload ({iters} iterations each), "
                      f"mean wall time per solve incl. setup"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    A, b, cfg, desc = _workload(args.workload)
    from oracle import oracle as O
    ref = O.reference()
    kind = "reference" if ref is not None else "port"
    which = "ref" if ref is not None else "port"
    cores = os.cpu_count() or 1
    if ref is not None:
        ref.ref_set_threads(cores)
    else:
        cores = 1
    c = O.default_config(use_abmc=int(cfg["use_abmc"]), max_iterations=cfg["maxiter"], tolerance=cfg["tol"],
                         shift_parameter=cfg["shift"], abmc_block_size=cfg["abmc_block_size"],
                         abmc_num_colors=cfg["abmc_num_colors"])
    for _ in range(args.warmup):
        O.solve(A, b, cfg["method"], c, which=which)
    times = []
    iters = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, r, _ = O.solve(A, b, cfg["method"], c, which=which)
        times.append(time.perf_counter() - t0)
        iters = r.iterations
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(desc, iterations=iters),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"{args.steps} full solves, reference headers on {cores} OpenMP threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ncu_case(args):
    import numpy as np

    import sparsesolv_ngsolve as ss
    A, b, cfg, desc = _workload(args.workload)
    s = ss.SparseSolvSolver(A, method=cfg["method"], tol=cfg["tol"], maxiter=cfg["maxiter"], shift=cfg["shift"],
                            use_abmc=cfg["use_abmc"], abmc_block_size=cfg["abmc_block_size"],
                            abmc_num_colors=cfg["abmc_num_colors"])
    x = np.zeros_like(b)
    r = s.Solve(b, x)
    print(json.dumps({"ncu_case": args.workload, "iterations": r.iterations, "converged": r.converged,
                      "kernels": r.kernel_launches}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="iccg64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run exactly one solve of the workload and exit (for ncu captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ids = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = ids[local]

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.ncu_case:
        return run_ncu_case(args)

    import numpy as np
    import torch

    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    dev = torch.device("cuda:0")

    A, b, cfg, desc = _workload(args.workload)
    lib = _capi.load()
    mat = ss._Matrix(A)
    n = A.shape[0]
    d_b = torch.from_numpy(b).to(dev)
    d_x = torch.zeros(n, dtype=torch.float64, device=dev)
    c = _capi.default_config(tolerance=cfg["tol"], max_iterations=cfg["maxiter"], shift_parameter=cfg["shift"],
                             use_abmc=cfg["use_abmc"], abmc_block_size=cfg["abmc_block_size"],
                             abmc_num_colors=cfg["abmc_num_colors"])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def solve_dev(keep=None):
        h = ctypes.c_void_p()
        _capi.check(lib.ssv_solver_create(mat.h, None, ctypes.byref(h)))
        d_x.zero_()
        res = _capi.ssv_result()
        _capi.check(lib.ssv_solver_solve_dev(h, cfg["method"].encode(), ctypes.byref(c),
                                             ctypes.c_void_p(d_b.data_ptr()), ctypes.c_void_p(d_x.data_ptr()),
                                             ctypes.byref(res), None, 0))
        if keep is None:
            lib.ssv_solver_destroy(h)
        else:
            keep.append(h)
        return res

    for _ in range(args.warmup):
        solve_dev()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, launches, iters, conv = [], 0, 0, True
    setup_s, solve_s = [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        r = solve_dev()
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        launches += r.kernel_launches
        setup_s.append(r.setup_seconds)
        solve_s.append(r.solve_seconds)
        iters = r.iterations
        conv = conv and bool(r.converged)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clock_info = clocks.stop()
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = ms_per_step / 1e3

    # warm variant: ordering / graph caches of the same solver object reused
    keep = []
    solve_dev(keep)
    hwarm = keep[0]
    warm_ms = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        d_x.zero_()
        res = _capi.ssv_result()
        e0.record()
        _capi.check(lib.ssv_solver_solve_dev(hwarm, cfg["method"].encode(), ctypes.byref(c),
                                             ctypes.c_void_p(d_b.data_ptr()), ctypes.c_void_p(d_x.data_ptr()),
                                             ctypes.byref(res), None, 0))
        e1.record()
        torch.cuda.synchronize()
        warm_ms.append(e0.elapsed_time(e1))
    # per-phase roofline of one iteration on the warm handle
    prof = _capi.ssv_phase_profile()
    _capi.check(lib.ssv_solver_profile(hwarm, cfg["method"].encode(), ctypes.byref(c), 200, ctypes.byref(prof)))
    phases = prof.as_list()
    lib.ssv_solver_destroy(hwarm)
    peak, peak_kind = _peaks()
    iter_ms = sum(p["ms"] for p in phases)
    dom = max(phases, key=lambda p: p["ms"])
    achieved = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": dom["name"], "peak_kind": peak_kind,
                "phases": [{**p, "GBps": p["bytes"] / (p["ms"] * 1e-3) / 1e9} for p in phases],
                "iteration_ms": iter_ms,
                "iteration_GBps": sum(p["bytes"] for p in phases) / (iter_ms * 1e-3) / 1e9}

    # end to end through the public API with host buffers
    solver = ss.SparseSolvSolver(A, method=cfg["method"], tol=cfg["tol"], maxiter=cfg["maxiter"],
                                 shift=cfg["shift"], use_abmc=cfg["use_abmc"],
                                 abmc_block_size=cfg["abmc_block_size"], abmc_num_colors=cfg["abmc_num_colors"])
    xh = np.zeros(n)
    for _ in range(2):
        xh[:] = 0
        solver.Solve(b, xh)
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        xh[:] = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        rr = solver.Solve(b, xh)
        e1.record()
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    true_res = float(np.linalg.norm(b - A @ xh) / np.linalg.norm(b))
    h2d = A.nnz * 8 + 2 * n * 8
    d2h = n * 8 + 64

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(desc, iterations=iters, converged=conv, parallelism=f"replicas{world}",
                           l2="flushed between timed steps (256 MB write)",
                           cold_setup_s=statistics.mean(setup_s), cold_iterate_s=statistics.mean(solve_s),
                           warm_time_to_solution_s=statistics.mean(warm_ms) / 1e3,
                           ms_per_iter_warm=statistics.mean(warm_ms) / max(iters, 1),
                           true_rel_residual=true_res),
            "e2e": {"value": statistics.mean(e2e_ms) / 1e3, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": roofline, "gpu_launches": int(launches), "clocks": clock_info}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(A, b, cfg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del solver
    mat = None
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
