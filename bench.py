"""Benchmark of the B200 solve path (one JSON line on rank 0).

Default workload ``ams40``: real magnetostatic curl-curl on a Kuhn 6-tet mesh
of a 40^3 unit cube (462,520 HCurl edges, 7,432,120 nonzeros, 68,921
vertices; nu = 1, iron block nu = 1e-3, 1e-6 nu M mass term, Dirichlet
boundary, square loop source), Compact AMS preconditioner + CG to 1e-10. One
step = one PCG solve to tolerance with the preconditioner built, the matrix,
b and x resident in HBM; metric = time-to-solution (s), lower is better. The
line's value is the FP32-preconditioner (mixed) form (nodal V-cycles through
the fused level products); the plain FP64 form is measured in the same run
(config.plain_fp64), and the batched form on the
40^3 complex eddy-current family (8 frequencies x 4 right-hand sides, one
launch graph) is measured against 32 sequential FP64 solves
(config.batched_family) unless --no-extras.

``--workload iccg64``: the plain FP64 ICCG drop-in on the 64^3 7-point
Laplacian (a complete SparseSolvSolver.Solve per step, set-up included).
``--workload eddy64``: the complex eddy-current system on the 64^3 Kuhn mesh
(1,872,064 complex edge unknowns), ComplexCompactAMS + COCR to 1e-10, plain
FP64; its CPU baseline is a bounded sample of COCR iterations of the
restatement, extrapolated to the full iteration count.

``--impl reference`` times the reference's CPU implementation of the same
workload on the host cores: for ICCG its own headers (oracle/_ref); for the
AMS workloads the reference's AMS needs NGSolve, so the C++ restatement in
oracle/ (OpenMP over all host cores) stands in. Multi-GPU: independent
replicas (one per rank, no collective on the data path), max over ranks.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "ngsolve-sparsesolv_b200"))

METRIC = "time-to-solution @1e-10 (s), ms/iter, SpMV HBM GB/s: mixed/batched vs plain FP64 GPU"
UNIT = "s"
# dram__bytes_read.sum + dram__bytes_write.sum of one eddy64 fine-residual launch (ncu; None until captured)
# DRAM bytes per launch of the fine residual at 64^3: the 48^3 ncu capture's traffic (195.3 MB against
# 195.2 MB algorithmic) scaled to 64^3 by the algorithmic bytes (461.3 MB)
EDDY_FINE_RESIDUAL_TRAFFIC = 461.5e6
# COCR iterations in each timed step of the reference arm on eddy64 (a bounded sample)
REF_SAMPLE_ITERS = 20


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"



def _init_dist(world, backend="nccl"):
    """One process group for the replicas (None on one rank); a short timeout, so ranks
    that wait for a missing peer end with an error."""
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def _max_over_ranks(value, dist, device):
    """The job's time: the maximum of the ranks' values (every rank calls this once)."""
    if not dist:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
    import torch

    import sparsesolv_ngsolve as ss
    if args.workload == "eddy64":
        # one warm solve first (tuner, graph capture), then the profiled one inside the NVTX
        # range "solve" (capture with ncu --nvtx --nvtx-include "solve/"; SSV_GRAPH_MODE=chunk)
        d = _eddy_system(args.eddy_nc)
        pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"],
                                                 coord_x=d["coords"][0], coord_y=d["coords"][1],
                                                 coord_z=d["coords"][2], precision=args.precision_eddy)
        inv = (ss.MixedCOCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=EDDY_MAXITER, tol=1e-10,
                                  restart_drop=REFINE_DROP) if args.precision_eddy != "fp64" else
               ss.COCRSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=EDDY_MAXITER, tol=1e-10))
        inv * d["f"]
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("solve")
        inv * d["f"]
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"ncu_case": args.workload, "mesh": f"{args.eddy_nc}^3", "precision": args.precision_eddy,
                          "iterations": inv.iterations}))
        if args.profile_levels:  # per-level V-cycle times (warm, back to back) of every subspace
            for sub in range(4):
                rows, last = pre.profile_levels(sub, reps=20)
                print(json.dumps({"subspace": sub, "levels": [{"level": l, "R_us": r * 1e3, "U_us": u * 1e3,
                                                               "R_shape": sr, "U_shape": su}
                                                              for l, r, u, sr, su in rows],
                                  "last_step_us": last * 1e3}))
        return
    if args.workload == "batched40":
        # the 40^3 eddy family (8 frequencies x 4 sources) in one batched COCR solve, FP64
        # preconditioners; one warm solve (tuners, graph), then the profiled one in "solve"
        from sparsesolv_ngsolve import hcurl as H
        d = H.eddy_family(args.family_nc, nrhs=4)
        pres = [ss.ComplexCompactAMSPreconditioner(a, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                                   coord_y=d["coords"][1], coord_z=d["coords"][2])
                for a in d["a_real"]]
        bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=1000,
                                  tol=1e-10)
        d_B = torch.from_numpy(np.ascontiguousarray(d["B"]).view(np.float64).reshape(-1)).cuda()
        d_X = torch.zeros_like(d_B)
        bs.solve_dev(d_B.data_ptr(), d_X.data_ptr())
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("solve")
        bs.solve_dev(d_B.data_ptr(), d_X.data_ptr())
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"ncu_case": args.workload, "mesh": f"{args.family_nc}^3",
                          "systems": int(d["B"].shape[0] * d["B"].shape[1]),
                          "max_iterations": int(bs.iterations.max())}))
        return
    if args.workload == "ams40":
        d = _ams_system()
        pre = _ams_pre(ss, d, args.precision)
        inv = ss.PCGSolver(d["A"], pre, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
        x = np.zeros(d["A"].shape[0])
        r = inv.Solve(d["f"], x)
        print(json.dumps({"ncu_case": args.workload, "precision": args.precision, "iterations": r.iterations,
                          "converged": r.converged, "kernels": r.kernel_launches}))
        return
    A, b, cfg, desc = _workload(args.workload)
    s = ss.SparseSolvSolver(A, method=cfg["method"], tol=cfg["tol"], maxiter=cfg["maxiter"], shift=cfg["shift"],
                            use_abmc=cfg["use_abmc"], abmc_block_size=cfg["abmc_block_size"],
                            abmc_num_colors=cfg["abmc_num_colors"])
    x = np.zeros_like(b)
    r = s.Solve(b, x)
    print(json.dumps({"ncu_case": args.workload, "iterations": r.iterations, "converged": r.converged,
                      "kernels": r.kernel_launches}))


# ---------------------------------------------------------------------------
# AMS workloads
# ---------------------------------------------------------------------------
AMS_DESC = {"workload": "ams40: real magnetostatic curl-curl, Kuhn 6-tet mesh of a 40^3 cube (462,520 edges, "
                        "7,432,120 nnz, 68,921 vertices), nu=1 / iron 1e-3, 1e-6 nu M, Compact AMS (cycle 1) + CG, "
                        "tol 1e-10",
            "tol": 1e-10, "rhs": "square loop current at mid-height (discretely divergence-free)"}


def _ams_system():
    from sparsesolv_ngsolve import hcurl as H
    return H.magnetostatic(40)


def _ams_pre(ss, d, precision):
    return ss.CompactAMSPreconditioner(d["A"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                       coord_y=d["coords"][1], coord_z=d["coords"][2], precision=precision)


def cpu_baseline_ams(d, budget_s=20.0):
    """The AMS restatement (oracle/, NGSolve being absent) + sparsesolv::CGSolver on all host cores."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.AmsOracle.set_threads(cores)
    t0 = time.perf_counter()
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"])
    setup = time.perf_counter() - t0
    cfg = O.default_config(tolerance=1e-10, max_iterations=500)
    times, iters = [], 0
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        _, r, _ = o.pcg(d["f"], config=cfg)
        times.append(time.perf_counter() - t0)
        iters = r.iterations
        if time.perf_counter() > t_end or len(times) >= 10:
            break
    return {"value": statistics.mean(times), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(times)} full PCG solves of the workload ({iters} iterations each) with the AMS "
                      f"restatement on {cores} OpenMP threads; mean wall time per solve, preconditioner built "
                      f"(its set-up took {setup:.2f} s)"}


def run_reference_ams(args, rank, world):
    if rank != 0:
        return
    d = _ams_system()
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.AmsOracle.set_threads(cores)
    o = O.AmsOracle(d["A"], d["G"], d["freedofs"], *d["coords"])
    cfg = O.default_config(tolerance=1e-10, max_iterations=500)
    for _ in range(args.warmup):
        o.pcg(d["f"], config=cfg)
    times, iters = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, r, _ = o.pcg(d["f"], config=cfg)
        times.append(time.perf_counter() - t0)
        iters = r.iterations
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(AMS_DESC, iterations=iters, ms_per_iter=v * 1e3 / max(iters, 1)),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} full PCG solves with the AMS restatement on {cores} OpenMP "
                                       f"threads (the reference's AMS needs NGSolve, absent here)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ams(args, rank, world, local):
    import numpy as np
    import torch

    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi

    dist = _init_dist(world)
    torch.cuda.set_device(0)
    dev = torch.device("cuda:0")
    lib = _capi.load()
    d = _ams_system()
    A = d["A"]
    n = A.shape[0]
    mat = ss._Matrix(A)
    d_fd = torch.from_numpy(np.ascontiguousarray(d["freedofs"].astype(np.uint8))).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(d["f"])).to(dev)
    d_x = torch.zeros(n, dtype=torch.float64, device=dev)
    cfg = _capi.default_config(tolerance=1e-10, max_iterations=500)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev).fill_(1.0)  # > 126 MB L2
    t0 = time.perf_counter()
    pre = _ams_pre(ss, d, "fp64")
    setup_s = time.perf_counter() - t0

    def solve_dev():
        d_x.zero_()
        res = _capi.ssv_result()
        _capi.check(lib.ssv_pcg_solve_dev(mat.h, pre._h, ctypes.cast(d_fd.data_ptr(), _capi.PU8), ctypes.byref(cfg),
                                          ctypes.c_void_p(d_b.data_ptr()), ctypes.c_void_p(d_x.data_ptr()),
                                          ctypes.byref(res), None, 0))
        return res

    def timed_steps(k):
        ms, launches, iters, conv = [], 0, 0, True
        for _ in range(k):
            _l2_evict(flush)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            r = solve_dev()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            launches += r.kernel_launches
            iters = r.iterations
            conv = conv and bool(r.converged)
        return ms, launches, iters, conv

    def true_res():
        x = d_x.cpu().numpy()
        fd = d["freedofs"].astype(bool)
        return float(np.linalg.norm((d["f"] - A @ np.where(fd, x, 0))[fd]) / np.linalg.norm(d["f"]))

    forms = {}
    for prec in ("fp64", "fp32"):
        pre.precision = prec
        for _ in range(args.warmup):
            solve_dev()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        clocks = ClockSampler(local)
        clocks.start()
        ms, launches, iters, conv = timed_steps(args.steps)
        clock_info = clocks.stop()
        total_ms = sum(ms)
        total_ms = _max_over_ranks(total_ms, dist, dev)
        prof = pre.profile(nrhs=1, reps=20)
        prof_cold = pre.profile(nrhs=1, reps=10, cold=True)
        forms[prec] = {"ms_per_step": total_ms / args.steps, "launches": launches, "iterations": iters,
                       "converged": conv, "clocks": clock_info, "phases": prof, "phases_cold": prof_cold,
                       "true_rel_residual": true_res(), "x": d_x.cpu().numpy()}
    peak, peak_kind = _peaks()
    # headline: the mixed form (FP32 subspace hierarchies, the faster form here);
    # the plain FP64 form is reported beside it
    mixed, plain = forms["fp32"], forms["fp64"]
    head = mixed

    def gbps(p):
        return p["bytes"] / (p["ms"] * 1e-3) / 1e9

    def phase(form, name):
        return next(p for p in form["phases"] if p["name"] == name)

    def phase_cold(form, name):
        return next(p for p in form["phases_cold"] if p["name"] == name)

    # the fine-level residual SpMV, each launch timed alone after an L2 flush
    # (A_bc is 89 MB: back to back it would be served partly from L2)
    spmv = phase_cold(head, "fine_residual")
    spmv_warm = phase(head, "fine_residual")
    achieved = gbps(spmv)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": 105.2e6,
                "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of one launch of this kernel "
                                "(ncu --set full, same workload, mean of 2 launches), per launch; the sliced-ELL "
                                "copy's padding (2.9% of the entries) and row map add 3% to the algorithmic bytes",
                "kernel": "k_sell_spmv fine residual (A_bc in 32-row sliced-ELL, 7.43M nnz, FP64; the shape tuner "
                          "keeps it where it times faster than the CSR shapes, on every B200 run so far), "
                          "each launch timed alone after evicting L2 by reading a 256 MB buffer (a write-based "
                          "flush leaves dirty lines whose write-back the launch would pay for: "
                          "SSV_PROFILE_FLUSH=write measures that form)",
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": spmv["bytes"], "launch_ms": spmv["ms"],
                "warm_GBps": gbps(spmv_warm),
                "phases_cold": [{**p, "GBps": gbps(p)} for p in head["phases_cold"]],
                "phases": [{**p, "GBps": gbps(p)} for p in head["phases"]],
                "phases_plain_fp64": [{**p, "GBps": gbps(p)} for p in plain["phases"]]}
    fdm = d["freedofs"].astype(bool)
    xm, xp = mixed["x"], plain["x"]
    e = np.where(fdm, xm - xp, 0)
    xp0 = np.where(fdm, xp, 0)
    err_energy = float(np.sqrt(abs(e @ (A @ e))) / np.sqrt(abs(xp0 @ (A @ xp0))))

    # end to end through the public API with host buffers (the headline form)
    pre.precision = "fp32"
    solver = ss.PCGSolver(A, pre, freedofs=d["freedofs"], maxiter=500, tol=1e-10)
    xh = np.zeros(n)
    for _ in range(2):
        xh[:] = 0
        solver.Solve(d["f"], xh)
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        _l2_evict(flush)
        xh[:] = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.Solve(d["f"], xh)
        e1.record()
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    value = head["ms_per_step"] / 1e3
    config = dict(AMS_DESC, parallelism=f"replicas{world}", l2="evicted between timed steps (256 MB read)",
                  form="mixed: FP32 subspace AMG hierarchies (diagonally scaled); the three nodal V-cycles "
                       "through the fused level products (down b' = R b, up x = U [b; e]: two launches per level), "
                       "the gradient V-cycle in four passes (fused, it loses too much in FP32); FP64 fine level in "
                       "its sliced-ELL copy, transfers, coarsest LDL^T solves and CG",
                  iterations=head["iterations"], converged=head["converged"],
                  ms_per_iter=head["ms_per_step"] / max(head["iterations"], 1),
                  spmv_GBps=achieved, true_rel_residual=head["true_rel_residual"],
                  error_vs_fp64_energy_norm=err_energy,
                  plain_fp64={"form": "FP64 subspace AMG hierarchies, every V-cycle through the fused level "
                                      "products",
                              "time_to_solution_s": plain["ms_per_step"] / 1e3, "iterations": plain["iterations"],
                              "ms_per_iter": plain["ms_per_step"] / max(plain["iterations"], 1),
                              "true_rel_residual": plain["true_rel_residual"]},
                  speedup_mixed_vs_plain=plain["ms_per_step"] / mixed["ms_per_step"],
                  ams_setup_s=setup_s)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 Krylov + f32 preconditioner hierarchy",
            "data": "synthetic", "config": config,
            "e2e": {"value": statistics.mean(e2e_ms) / 1e3, "unit": UNIT,
                    # b and x, the FreeDofs mask, and the matrix values, which Solve re-reads from the
                    # host matrix every call (the matrix may have been modified in place)
                    "h2d_bytes_per_step": int(2 * n * 8 + n + A.nnz * 8),
                    "d2h_bytes_per_step": int(n * 8 + 64)},
            "roofline": roofline, "gpu_launches": int(head["launches"]), "clocks": head["clocks"]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_ams(d)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del solver
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Complex eddy current at 64^3 (ComplexCompactAMS + COCR): the default workload
# ---------------------------------------------------------------------------
EDDY_DESC = {"workload": "eddy64: complex eddy current A = K + j omega sigma M_cond, Kuhn 6-tet mesh of a 64^3 cube "
                         "(1,872,064 edges, 30,331,072 nnz, complex<double>), omega = 2 pi 3e4, sigma = 5.8e7 in a "
                         "copper annulus, nu_r = 1e-3 core, auxiliary K + |omega| sigma M + 1e-6 nu M, "
                         "ComplexCompactAMS (cycle 1) + COCR, tol 1e-10",
             "tol": 1e-10, "rhs": "square loop currents at mid-height (discretely divergence-free)"}
REFINE_DROP = 1e-5
EDDY_MAXITER = 3000


def _eddy_system(nc=64):
    from sparsesolv_ngsolve import hcurl as H
    return H.eddy_current(nc)


def _rel_err(x, xref):
    return float(np.linalg.norm(x - xref) / max(np.linalg.norm(xref), 1e-300))


def _eddy_true_res(d, x):
    fdm = d["freedofs"].astype(bool)
    return float(np.linalg.norm((d["f"] - d["A"] @ np.where(fdm, x, 0))[fdm]) / np.linalg.norm(d["f"][fdm]))


def cpu_eddy_full(d):
    """One full solve of the workload with the ComplexCompactAMS restatement +
    COCRSolverNGS on all host cores (NGSolve, which the reference's AMS needs,
    is absent); returns the baseline record and the solution."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.AmsOracle.set_threads(cores)
    t0 = time.perf_counter()
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    x, its, _ = o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=EDDY_MAXITER, tol=1e-10)
    wall = time.perf_counter() - t0
    rec = {"value": wall, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"1 full COCR solve of the workload ({int(its)} iterations, {wall / max(int(its), 1) * 1e3:.1f} "
                     f"ms per iteration) with the ComplexCompactAMS restatement on {cores} OpenMP threads, "
                     f"preconditioner built (its set-up took {setup:.1f} s)",
           "iterations": int(its), "true_rel_residual": _eddy_true_res(d, x), "setup_s": setup}
    return rec, x


def run_reference_eddy(args, rank, world):
    if rank != 0:
        return
    d = _eddy_system()
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    O.AmsOracle.set_threads(cores)
    o = O.AmsOracle(d["a_real"], d["G"], d["freedofs"], *d["coords"])
    for _ in range(args.warmup):  # warm-up: bounded samples (5 COCR iterations), untimed
        o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=5, tol=1e-10)
    # one full solve to tolerance, untimed: its iteration count scales the samples below
    t0 = time.perf_counter()
    x, its, _ = o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=EDDY_MAXITER, tol=1e-10)
    full_s = time.perf_counter() - t0
    iters = int(its)
    sample = min(REF_SAMPLE_ITERS, max(iters, 1))
    times = []
    for _ in range(args.steps):  # every timed step: a bounded sample of `sample` COCR iterations
        t0 = time.perf_counter()
        o.cocr(d["A"], d["f"], freedofs=d["freedofs"], maxiter=sample, tol=1e-10)
        times.append((time.perf_counter() - t0) * iters / sample)
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": dict(EDDY_DESC, iterations=iters, ms_per_iter=v * 1e3 / max(iters, 1),
                           true_rel_residual=_eddy_true_res(d, x), full_solve_s=full_s,
                           value_is=f"time to solution: each step's {sample}-iteration sample scaled to the full "
                                    f"solve's {iters} iterations (the full solve, run once untimed, took "
                                    f"{full_s:.1f} s)"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} samples of {sample} COCR iterations each, scaled to the "
                                       f"{iters} iterations of one full solve, with the ComplexCompactAMS "
                                       f"restatement on {cores} OpenMP threads; warm-up steps are 5-iteration "
                                       f"samples"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _l2_evict(buf):
    """Evicts L2 by reading a buffer larger than it (a read leaves clean lines:
    no write-back for the next kernel to pay)."""
    import torch
    buf.sum()
    torch.cuda.synchronize()


def batched_family_extra(ss, nc=40):
    """Config 4: the 40^3 eddy-current family, 8 frequencies x 4 sources (32
    systems). The mixed batched form (ComplexCompactAMS per frequency with its
    nodal hierarchies in FP32, refined COCR cycles to a true residual of 1e-10, one launch
    graph with the autotuned SpMM) against 32 sequential plain FP64 GPU solves
    (COCRSolver, FP64 ComplexCompactAMS); the FP64 batched form beside it.
    Device time (CUDA events), inputs resident in HBM."""
    import torch

    from oracle import oracle as O
    from sparsesolv_ngsolve import _capi
    from sparsesolv_ngsolve import hcurl as H
    lib = _capi.load()
    dev = torch.device("cuda:0")
    d = H.eddy_family(nc, nrhs=4)
    F, R, n = len(d["omegas"]), 4, d["K"].shape[0]
    fdm = d["freedofs"].astype(bool)
    pres = [ss.ComplexCompactAMSPreconditioner(a, d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                               coord_y=d["coords"][1], coord_z=d["coords"][2])
            for a in d["a_real"]]
    d_B = torch.from_numpy(np.ascontiguousarray(d["B"]).view(np.float64).reshape(-1)).to(dev)
    d_X = torch.zeros_like(d_B)

    def tres(f, x, b):
        return float(np.linalg.norm((b - d["A"][f] @ np.where(fdm, x, 0))[fdm]) / np.linalg.norm(b[fdm]))

    def timed(fn, reps=2):
        fn()
        out = []
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / 1e3)
        return min(out)

    # 32 sequential plain FP64 solves (the drop-in, one system at a time)
    mats = [ss._Matrix(a) for a in d["A"]]
    d_fd = torch.from_numpy(np.ascontiguousarray(d["freedofs"].astype(np.uint8))).to(dev)
    d_b1 = torch.zeros(2 * n, dtype=torch.float64, device=dev)
    d_x1 = torch.zeros(2 * n, dtype=torch.float64, device=dev)
    seq_x = np.zeros_like(d["B"])
    its_seq = np.zeros((F, R), np.int32)

    def seq_all(keep=False):
        it = ctypes.c_int32()
        for f in range(F):
            for r in range(R):
                d_b1.copy_(d_B.view(F, R, 2 * n)[f, r])
                _capi.check(lib.ssv_cocr_solve_dev(mats[f].h, pres[f]._h, ctypes.cast(d_fd.data_ptr(), _capi.PU8),
                                                   1000, 1e-10, 0, ctypes.c_void_p(d_b1.data_ptr()),
                                                   ctypes.c_void_p(d_x1.data_ptr()), ctypes.byref(it)))
                if keep:
                    seq_x[f, r] = d_x1.cpu().numpy().view(np.complex128)
                    its_seq[f, r] = it.value
    seq_all(keep=True)
    t_seq = timed(seq_all, reps=1)
    out = {"family": f"complex eddy current on the {nc}^3 Kuhn mesh ({n} edges), 8 frequencies 1 kHz..100 kHz x 4 "
                     f"loop sources (default_rng(1)), ComplexCompactAMS per frequency + COCR, tol 1e-10",
           "sequential_fp64_s": t_seq, "iterations_sequential": its_seq.ravel().tolist(),
           "max_true_residual_sequential": max(tres(f, seq_x[f, r], d["B"][f, r]) for f in range(F) for r in range(R))}
    # batched, FP64 preconditioners, the reference recurrence per column
    bs = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=1000,
                              tol=1e-10)
    out["batched_fp64_s"] = timed(lambda: bs.solve_dev(d_B.data_ptr(), d_X.data_ptr()))
    X = d_X.cpu().numpy().view(np.complex128).reshape(F, R, n)
    out["iterations_batched_fp64"] = bs.iterations.ravel().tolist()
    out["max_true_residual_batched_fp64"] = max(tres(f, X[f, r], d["B"][f, r]) for f in range(F) for r in range(R))
    del bs
    # the mixed batched form
    for p in pres:
        p.precision = "fp32_nodal"
    bm = ss.BatchedCOCRSolver(d["K"], d["M"], d["omegas"], pres, nrhs=4, freedofs=d["freedofs"], maxiter=1500,
                              tol=1e-10, restart_drop=REFINE_DROP)
    out["batched_mixed_s"] = timed(lambda: bm.solve_dev(d_B.data_ptr(), d_X.data_ptr()))
    tm = bm.last_timing
    X = d_X.cpu().numpy().view(np.complex128).reshape(F, R, n)
    out.update({"iterations_batched_mixed": bm.iterations.ravel().tolist(), "batched_mixed_cycles": tm["cycles"],
                "batched_mixed_kernel_launches": tm["kernel_launches"],
                "max_true_residual_batched_mixed": max(tres(f, X[f, r], d["B"][f, r])
                                                       for f in range(F) for r in range(R)),
                "batched_mixed_all_converged": bool(bm.converged.all()),
                "max_error_mixed_vs_sequential_fp64": max(_rel_err(X[f, r], seq_x[f, r])
                                                          for f in range(F) for r in range(R)),
                "autotuned_spmm": bm.tuning["chosen"]})
    out["speedup_batched_mixed_vs_sequential_fp64"] = t_seq / out["batched_mixed_s"]
    out["speedup_batched_fp64_vs_sequential_fp64"] = t_seq / out["batched_fp64_s"]
    # two columns against the FP64 restatement (the lowest and highest frequency)
    O.AmsOracle.set_threads(os.cpu_count() or 1)
    errs = []
    for f in (0, F - 1):
        o = O.AmsOracle(d["a_real"][f], d["G"], d["freedofs"], *d["coords"])
        xo, _, _ = o.cocr(d["A"][f], d["B"][f, 0], freedofs=d["freedofs"], maxiter=1000, tol=1e-10)
        errs.append(_rel_err(X[f, 0], xo))
    out["error_mixed_vs_reference_f0_f7"] = errs
    del bm
    for p in pres:
        p.precision = "fp64"
    return out


def run_eddy(args, rank, world, local):
    import torch

    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi

    dist = _init_dist(world)
    torch.cuda.set_device(0)
    dev = torch.device("cuda:0")
    lib = _capi.load()
    d = _eddy_system()
    A = d["A"]
    n = A.shape[0]
    mat = ss._Matrix(A)
    d_fd = torch.from_numpy(np.ascontiguousarray(d["freedofs"].astype(np.uint8))).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(d["f"]).view(np.float64)).to(dev)
    d_x = torch.zeros(2 * n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev).fill_(1.0)  # > 126 MB L2
    t0 = time.perf_counter()
    pre = ss.ComplexCompactAMSPreconditioner(d["a_real"], d["G"], freedofs=d["freedofs"], coord_x=d["coords"][0],
                                             coord_y=d["coords"][1], coord_z=d["coords"][2])
    setup_s = time.perf_counter() - t0
    setup_times = pre.setup_times
    fdp = ctypes.cast(d_fd.data_ptr(), _capi.PU8)
    info = _capi.ssv_refine_info()
    nl = ctypes.c_int64()

    def solve_plain():
        its = ctypes.c_int32()
        _capi.check(lib.ssv_cocr_solve_dev(mat.h, pre._h, fdp, EDDY_MAXITER, 1e-10, 0, ctypes.c_void_p(d_b.data_ptr()),
                                           ctypes.c_void_p(d_x.data_ptr()), ctypes.byref(its)))
        return its.value, 1

    def solve_mixed():
        _capi.check(lib.ssv_cocr_refined_solve_dev(mat.h, pre._h, fdp, EDDY_MAXITER, 1e-10, REFINE_DROP, 0,
                                                   ctypes.c_void_p(d_b.data_ptr()), ctypes.c_void_p(d_x.data_ptr()),
                                                   ctypes.byref(info)))
        return info.iterations, info.cycles

    def timed_form(fn, sample_clocks):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        clocks = ClockSampler(local) if sample_clocks else None
        if clocks:
            clocks.start()
        ms, iters, cycles, launches = [], 0, 0, 0
        for _ in range(args.steps):
            _l2_evict(flush)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            iters, cycles = fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            _capi.check(lib.ssv_cocr_last_launches(ctypes.byref(nl)))
            launches += nl.value
        clock_info = clocks.stop() if clocks else None
        total_ms = sum(ms)
        total_ms = _max_over_ranks(total_ms, dist, dev)
        x = d_x.cpu().numpy().view(np.complex128).copy()
        return {"s": total_ms / args.steps / 1e3, "iterations": iters, "cycles": cycles, "launches": launches,
                "clocks": clock_info, "x": x, "true_rel_residual": _eddy_true_res(d, x)}

    plain = timed_form(solve_plain, True)
    prof = pre.profile(nrhs=1, reps=10)
    prof_cold = pre.profile(nrhs=1, reps=5, cold=True)
    # end to end through the public API with host buffers (the drop-in COCRSolver)
    inv = ss.COCRSolver(A, pre, freedofs=d["freedofs"], maxiter=EDDY_MAXITER, tol=1e-10)

    def e2e(solver, reps):
        solver * d["f"]
        out = []
        for _ in range(reps):
            _l2_evict(flush)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            solver * d["f"]
            e1.record()
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / 1e3)
        return statistics.mean(out)

    e2e_plain = e2e(inv, max(2, args.steps // 4))
    pre.precision = "fp32_nodal"
    mixed = timed_form(solve_mixed, False)
    invm = ss.MixedCOCRSolver(A, pre, freedofs=d["freedofs"], maxiter=EDDY_MAXITER, tol=1e-10,
                              restart_drop=REFINE_DROP)
    e2e_mixed = e2e(invm, max(2, args.steps // 4))
    prof_mixed = pre.profile(nrhs=1, reps=10)
    pre.precision = "fp64"
    peak, peak_kind = _peaks()

    def gbps(p):
        return p["bytes"] / (p["ms"] * 1e-3) / 1e9

    spmv = next(p for p in prof_cold if p["name"] == "fine_residual")
    spmv_warm = next(p for p in prof if p["name"] == "fine_residual")
    roofline = {"bound": "hbm", "achieved": gbps(spmv), "peak": peak, "unit": "GB/s", "frac": gbps(spmv) / peak,
                "traffic": EDDY_FINE_RESIDUAL_TRAFFIC,
                "traffic_note": "DRAM bytes of one launch of this kernel from an ncu capture on the 48^3 mesh "
                                "(dram__bytes.sum), scaled to 64^3 by the algorithmic bytes",
                "kernel": "k_sell_spmv fine residual (A_bc real in 32-row sliced-ELL, Re/Im columns, 30.3M nnz, FP64; "
                          "tuner-chosen over the CSR shapes), each launch timed alone after evicting L2 by reading a "
                          "256 MB buffer",
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": spmv["bytes"], "launch_ms": spmv["ms"],
                "warm_GBps": gbps(spmv_warm),
                "phases_cold": [{**p, "GBps": gbps(p)} for p in prof_cold],
                "phases": [{**p, "GBps": gbps(p)} for p in prof],
                "phases_mixed": [{**p, "GBps": gbps(p)} for p in prof_mixed]}
    value = plain["s"]
    config = dict(EDDY_DESC, parallelism=f"replicas{world}",
                  l2="evicted between timed steps (256 MB read)",
                  form="plain FP64 (the drop-in: COCRSolverNGS recurrence, FP64 ComplexCompactAMS)",
                  iterations=plain["iterations"], ms_per_iter=value * 1e3 / max(plain["iterations"], 1),
                  spmv_GBps=gbps(spmv), true_rel_residual=plain["true_rel_residual"],
                  true_rel_residual_meets_tol=bool(plain["true_rel_residual"] <= 1e-10),
                  stop_rule="plain form: the recurrence residual ||r_j|| / ||b|| <= tol (COCRSolverNGS, "
                            "sparsesolv_solvers.hpp:338-344), so its true residual can end above tol; mixed form: "
                            "the FP64 true residual <= tol",
                  ams_setup_s=setup_s, ams_setup_breakdown_s=setup_times,
                  mixed_form="ComplexCompactAMS with the three nodal hierarchies in FP32 (diagonally scaled) and the "
                             "gradient hierarchy, fine level, transfers and coarsest solves FP64, under refined COCR: "
                             f"cycles restarted from the FP64 true residual after a {REFINE_DROP:g} drop, stop on the "
                             "true residual",
                  mixed_time_to_solution_s=mixed["s"], mixed_iterations=mixed["iterations"],
                  mixed_cycles=mixed["cycles"], mixed_true_rel_residual=mixed["true_rel_residual"],
                  mixed_true_rel_residual_meets_tol=bool(mixed["true_rel_residual"] <= 1e-10),
                  mixed_ms_per_iter=mixed["s"] * 1e3 / max(mixed["iterations"], 1),
                  speedup_mixed_vs_plain=value / mixed["s"],
                  error_mixed_vs_plain=_rel_err(mixed["x"], plain["x"]),
                  e2e_mixed_s=e2e_mixed)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": config,
            "e2e": {"value": e2e_plain, "unit": UNIT,
                    # b and x, the FreeDofs mask, and the complex matrix values re-read every call
                    "h2d_bytes_per_step": int(2 * n * 16 + n + A.nnz * 16),
                    "d2h_bytes_per_step": int(n * 16)},
            "roofline": roofline, "gpu_launches": int(plain["launches"]), "clocks": plain["clocks"]}
    if rank == 0 and not args.no_extras:
        try:
            bf = batched_family_extra(ss)
            config["batched_family"] = bf
            for k in ("batched_mixed_s", "sequential_fp64_s", "batched_fp64_s",
                      "speedup_batched_mixed_vs_sequential_fp64", "speedup_batched_fp64_vs_sequential_fp64",
                      "max_true_residual_batched_mixed", "max_error_mixed_vs_sequential_fp64"):
                config[k] = bf[k]
        except Exception as exc:  # reported, not hidden
            config["batched_family"] = {"error": repr(exc)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, xref = cpu_eddy_full(d)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        config["reference_iterations"] = cb["iterations"]
        config["reference_true_rel_residual"] = cb["true_rel_residual"]
        config["reference_setup_s"] = cb["setup_s"]
        config["error_vs_reference"] = _rel_err(plain["x"], xref)
        config["mixed_error_vs_reference"] = _rel_err(mixed["x"], xref)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del inv, invm
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Nonlinear magnetostatic Newton sequence at 40^3 with the learned initial guess
# ---------------------------------------------------------------------------
NEWTON_DESC = {"workload": "newton40: nonlinear magnetostatics on the 40^3 Kuhn mesh (462,520 edges), iron nu(|B|) = "
                           "nu0 (k1 + k2 |B|^2), k1 = 1e-3, k2 = 5e-3, 20 Newton steps per load x 50 loads "
                           "(amplitudes U[0.5, 2], default_rng(2)), each step Update() + Compact AMS + CG to 1e-10; "
                           "per-edge MLP guess (12 features, 64 hidden, FP32, the library's own train/infer kernels) "
                           "trained on loads 0-29, judged on loads 30-49 against the previous-step guesses",
               "tol": 1e-10}


def run_newton(args, rank, world, local):
    import torch

    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import newton as NW
    if rank != 0:
        return
    torch.cuda.set_device(0)
    prob = NW.NonlinearMagnetostatic(40)
    amps = np.random.default_rng(2).uniform(0.5, 2.0, 50)
    nsteps = 20
    tm = {"update_s": 0.0, "solve_s": 0.0, "updates": 0, "solves": 0, "launches": 0}

    class TimedPre:
        """the AMS preconditioner, its Update() timed"""
        def __init__(self, J):
            t0 = time.perf_counter()
            self.p = ss.CompactAMSPreconditioner(J, prob.G, freedofs=prob.freedofs, coord_x=prob.coords[0],
                                                 coord_y=prob.coords[1], coord_z=prob.coords[2])
            self.create_s = time.perf_counter() - t0
            self._h = self.p._h

        def Update(self, J):
            t0 = time.perf_counter()
            self.p.Update(J)
            tm["update_s"] += time.perf_counter() - t0
            tm["updates"] += 1
            self._h = self.p._h

    class TimedSolver:
        def __init__(self, J, pre):
            self.inv = ss.PCGSolver(J, pre.p, freedofs=prob.freedofs, maxiter=500, tol=1e-10)

        def Solve(self, rhs, x):
            t0 = time.perf_counter()
            r = self.inv.Solve(rhs, x)
            tm["solve_s"] += time.perf_counter() - t0
            tm["solves"] += 1
            tm["launches"] += int(r.kernel_launches)
            return r

    t0 = time.perf_counter()
    tr = NW.run_loads(prob, amps[:30], nsteps, TimedPre, TimedSolver, collect=True)
    t_train_loads = time.perf_counter() - t0
    t0 = time.perf_counter()
    net, ys, loss = NW.train_predictor(tr)
    t_train = time.perf_counter() - t0
    ev = NW.run_loads(prob, amps[29:], nsteps, TimedPre, TimedSolver, predictor=net, scale=tr["scale"], yscale=ys)
    prev = int(sum(sum(x) for x in ev["iters_prev"][1:]))
    mlp = int(sum(sum(x) for x in ev["iters_mlp"][1:]))
    first = [int(x[0]) for x in ev["iters_prev"][1:]], [int(x[0]) for x in ev["iters_mlp"][1:]]
    per_step = (tm["update_s"] + tm["solve_s"]) / max(tm["solves"], 1)
    line = {"metric": METRIC, "value": per_step, "unit": UNIT, "n_gpus": world, "steps": tm["solves"], "warmup": 0,
            "ms_per_step": per_step * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (MLP f32)", "data": "synthetic",
            "config": dict(NEWTON_DESC, value_is="mean wall time of one Newton linear step: Update() + PCG solve",
                           update_s_mean=tm["update_s"] / max(tm["updates"], 1),
                           solve_s_mean=tm["solve_s"] / max(tm["solves"], 1), newton_steps=tm["solves"],
                           training_loads_wall_s=t_train_loads, mlp_training_s=t_train, mlp_last_loss=loss,
                           cg_iterations_eval_previous_step_guess=prev, cg_iterations_eval_learned_guess=mlp,
                           iteration_cut=1.0 - mlp / max(prev, 1),
                           first_step_iterations_previous=first[0], first_step_iterations_learned=first[1],
                           start_error_previous_mean=float(np.mean(ev["start_err_prev"])),
                           start_error_learned_mean=float(np.mean(ev["start_err_mlp"]))),
            "gpu_launches": tm["launches"],
            "gpu_launches_note": "kernels of the PCG solves (the set-up kernels of Update() are not counted)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="eddy64", choices=["eddy64", "ams40", "iccg64", "newton40", "batched40"],
                    help="batched40 (the 40^3 eddy family, batched COCR) is a --ncu-case only: its timed "
                         "figures are part of the eddy64 line")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched-family measurement")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"], help="AMS form of --ncu-case")
    ap.add_argument("--precision-eddy", default="fp64", choices=["fp64", "fp32_nodal", "fp32"],
                    help="AMS form of the eddy64 --ncu-case")
    ap.add_argument("--profile-levels", action="store_true",
                    help="with the eddy64 --ncu-case: print each subspace's per-level V-cycle times")
    ap.add_argument("--eddy-nc", type=int, default=64,
                    help="mesh size of the eddy64 --ncu-case (a smaller mesh for multi-pass ncu sections)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--family-nc", type=int, default=40, help="mesh of the batched40 --ncu-case (smaller for "
                                                                    "multi-pass captures)")
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

    if args.workload == "batched40" and not args.ncu_case:
        ap.error("--workload batched40 is an --ncu-case only (the batched family is timed in the eddy64 line)")
    if args.impl == "reference":
        if args.workload == "ams40":
            return run_reference_ams(args, rank, world)
        if args.workload == "eddy64":
            return run_reference_eddy(args, rank, world)
        return run_reference(args, rank, world)
    if args.ncu_case:
        return run_ncu_case(args)
    if args.workload == "ams40":
        return run_ams(args, rank, world, local)
    if args.workload == "eddy64":
        return run_eddy(args, rank, world, local)
    if args.workload == "newton40":
        return run_newton(args, rank, world, local)

    import numpy as np
    import torch

    import sparsesolv_ngsolve as ss
    from sparsesolv_ngsolve import _capi

    dist = _init_dist(world)
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
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev).fill_(1.0)  # > 126 MB L2

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
        _l2_evict(flush)
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
    total_ms = _max_over_ranks(total_ms, dist, dev)
    ms_per_step = total_ms / args.steps
    value = ms_per_step / 1e3

    # warm variant: ordering / graph caches of the same solver object reused
    keep = []
    solve_dev(keep)
    hwarm = keep[0]
    warm_ms = []
    for _ in range(max(3, args.steps // 2)):
        _l2_evict(flush)
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
        _l2_evict(flush)
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
                           l2="evicted between timed steps (256 MB read)",
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
