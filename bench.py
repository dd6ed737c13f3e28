"""Benchmark: MG-preconditioned CG time-to-solution on one B200 per rank.

Workload (default): 3D Poisson, continuous Q4, 64^3 uniform cells
(16,974,593 DoFs, 16,581,375 interior), f = 8 seeded sin modes, FP32
vertex-patch smoother / transfer / level operators inside the V-cycle under an
FP64 flexible CG, relative residual 1e-10.  A step is one complete solve from
x = 0 with the right-hand side resident in HBM.  The same solve with an FP64
V-cycle is timed beside it, and the mixed solution's error against that FP64
solve is reported.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 every rank solves its own seeded instance (independent problems, no
collective on the data path): value = total DoFs solved per second, timed as
the max over ranks.
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

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "MG-CG DoF/s to 1e-10 rel. residual, mixed vs plain FP64 on 1 B200; smoother GB/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson3d_q4_64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="solve", choices=["solve", "smoother", "operator"],
                    help="smoother / operator: only time the finest-level smoother "
                         "sweeps / FP64 operator applications (small commands for kernel "
                         "profiling)")
    ap.add_argument("--smoother", default="fp32", choices=["fp32", "tf32", "fp64"],
                    help="--mode smoother: FP32 SIMT kernel, tensor-core (TF32) kernel or FP64")
    return ap.parse_args()


def run_operator_only(args):
    """Times --steps finest-level FP64 operator applications (the CG's q = A p)
    after --warmup applications and prints one JSON line."""
    import torch
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    P = tps.PoissonProblem(dim, k, n)
    A = tps.LaplaceOperator(P)
    src = problems.make_rhs(args.workload)
    dst = torch.empty_like(src)
    for _ in range(args.warmup):
        A.vmult(dst, src)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(max(args.steps, 1)):
        A.vmult(dst, src)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"mode": "operator", "workload": args.workload, "ms_per_apply": ms,
                      "algorithmic_GBps": 2 * 8 * P.n_dofs() / (ms * 1e-3) / 1e9}), flush=True)
    P.close()


def run_smoother_only(args):
    """Times --steps sweeps of the finest-level smoother (8 colour launches
    each, --smoother precision) after --warmup sweeps and prints one JSON line."""
    import torch
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import _lib as L
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    P = tps.PoissonProblem(dim, k, n)
    lf = P.n_levels - 1
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    ms = ctypes.c_double()
    code = {"fp32": L.TPS_F32, "tf32": L.TPS_TF32, "fp64": L.TPS_F64}[args.smoother]
    if args.warmup > 0:
        L.check(L.lib().tps_time_smoother(P.handle, lf, code, args.warmup, ctypes.byref(ms), sp), P.handle)
    L.check(L.lib().tps_time_smoother(P.handle, lf, code, max(args.steps, 1), ctypes.byref(ms), sp), P.handle)
    total, per = smoother_bytes(dim, k, n, 8 if args.smoother == "fp64" else 4)
    print(json.dumps({"mode": "smoother", "smoother": args.smoother, "workload": args.workload,
                      "ms_per_sweep": ms.value, "algorithmic_GBps": total / (ms.value * 1e-3) / 1e9}),
          flush=True)
    P.close()


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def smoother_bytes(dim: int, k: int, n: int, s: int) -> tuple[int, list[int]]:
    """Algorithmic bytes of one coloured sweep: per colour, the union of the
    patch boxes of x is read, b is read on the union of patch interiors and x
    written there: s * (|U_c| + 2 |I_c|)."""
    per = []
    npd = n - 1
    for c in range(1 << dim):
        par = [(c >> d) & 1 for d in range(dim)]
        cnt = [((npd - p + 1) // 2 if npd > p else 0) for p in par]
        if 0 in cnt:
            per.append(0)
            continue
        u = 1
        for d in range(dim):
            first = par[d] * k
            last = (par[d] + 2 * (cnt[d] - 1)) * k + 2 * k
            u *= last - first + 1  # consecutive boxes touch: the union is an interval
        interior = 1
        for d in range(dim):
            interior *= cnt[d] * (2 * k - 1)
        per.append(s * (u + 2 * interior))
    return sum(per), per


def launches_per_solve(dim: int, n_levels: int, iterations: int) -> int:
    """Kernels of ours launched by one CG solve (the V-cycle is fixed; memsets excluded)."""
    colours = 1 << dim
    per_level = 2 * colours + 1 + (2 if dim == 3 else 1) * 2
    vcycle = per_level * (n_levels - 1) + 1  # coarse: the single patch (colour 0)
    init = 1 + 1 + 2 + vcycle + 2 + 1 + 2 + 1 + 1
    per_it = vcycle + 2 + 1 + 1 + 2 + 1 + 1
    return init + per_it * max(iterations - 1, 0)


def cpu_baseline(args, dim, k, n, its_full):
    """The CPU oracle (same algorithm: coloured patch smoother, FP32 V-cycle,
    FP64 flexible CG) on the host cores, on a bounded sample: the first m CG
    iterations of the same instance, scaled to the full iteration count."""
    import numpy as np
    from oracle import oracle as O
    from gputensorproductsmoother_b200 import problems, split_cells
    nc, nl = split_cells(n)
    b = problems.WORKLOADS[args.workload][3](dim, k, n, 0, "cpu").numpy()
    H = O.Hierarchy(dim, k, nc, nl)
    m = 1
    t0 = time.perf_counter()
    _, it, _ = H.solve_cg(b, precision=1, symmetric=True, rel_tol=1e-10, max_it=m)
    t = time.perf_counter() - t0
    # m iterations = (m + 1) V-cycles + m + 1 operator applications; scale per V-cycle
    t_full = t * (its_full + 1) / (m + 1)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    nint = (n * k - 1) ** dim
    return {"value": nint / t_full, "unit": "DoF/s", "cores": cores, "kind": "port",
            "sample": f"first {m} of {its_full} CG iterations of the same {n}^{dim} Q{k} "
                      f"instance ({t:.1f} s), scaled by V-cycle count"}, t


def run_reference(args):
    """Reference arm: the reference's CPU-runnable implementation of this
    path is the oracle port (the reference itself is GPU+deal.II only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    import numpy as np
    from oracle import oracle as O
    from gputensorproductsmoother_b200 import split_cells
    nc, nl = split_cells(n)
    b = problems.WORKLOADS[args.workload][3](dim, k, n, 0, "cpu").numpy()
    H = O.Hierarchy(dim, k, nc, nl)
    nint = (n * k - 1) ** dim
    # each step: one V-cycle-preconditioned CG iteration pair bounded to 1 iteration,
    # scaled to a full solve of `its` iterations
    x, its, _ = H.solve_cg(b, precision=1, symmetric=True, rel_tol=1e-10, max_it=1)
    its_full = 7
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        H.solve_cg(b, precision=1, symmetric=True, rel_tol=1e-10, max_it=1)
        t = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(t * (its_full + 1) / 2)
    ms = 1000 * statistics.mean(times)
    val = nint / (ms / 1000)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "DoF/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
            "data": "synthetic", "config": {"workload": args.workload, "dim": dim, "degree": k,
                                            "cells": n, "dofs": (n * k + 1) ** dim},
            "cpu_baseline": {"value": val, "unit": "DoF/s", "cores": cores, "kind": "port",
                             "sample": f"1 CG iteration (2 V-cycles) of the {n}^{dim} Q{k} "
                                       f"instance per step, scaled to {its_full} iterations"},
            "e2e": {"value": val, "unit": "DoF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args)
        return
    if args.mode == "smoother":
        run_smoother_only(args)
        return
    if args.mode == "operator":
        run_operator_only(args)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import _lib as L
    from gputensorproductsmoother_b200 import problems

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    dim, k, n, _ = problems.WORKLOADS[args.workload]
    P = tps.PoissonProblem(dim, k, n)
    S = tps.MultigridSolvers(P)
    b = problems.make_rhs(args.workload, seed=rank)
    x = torch.zeros_like(b)
    nint = problems.interior_dofs(dim, k, n)
    stream = torch.cuda.Stream()

    def solve(precision):
        x.zero_()
        _, rep = S.solve_cg(b, x, precision=precision, rel_tol=1e-10)
        return rep

    with torch.cuda.stream(stream):
        # FP64 reference solve (the FP64 GPU oracle solution) and its timing
        for _ in range(max(1, args.warmup // 2)):
            rep64 = solve("fp64")
        x64 = x.clone()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n64 = max(2, args.steps // 2)
        e0.record(stream)
        for _ in range(n64):
            rep64 = solve("fp64")
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1) / n64

        for _ in range(args.warmup):
            rep = solve("fp32")
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        clk.start()
        e0.record(stream)
        for _ in range(args.steps):
            rep = solve("fp32")
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = clk.stop()
        barrier()
        ms = e0.elapsed_time(e1) / args.steps
        err = (torch.linalg.norm(x - x64) / torch.linalg.norm(x64)).item()
        resid_check = rep.final_residual

        # dominant kernel: the FP32 fine-level smoother sweep (8 colour launches of
        # the TMA-staged kernel on the V-cycle's work vectors), CUDA events on `stream`
        lf = P.n_levels - 1
        msw = ctypes.c_double()
        sp = ctypes.c_void_p(stream.cuda_stream)
        L.check(L.lib().tps_time_smoother(P.handle, lf, L.TPS_F32, 3, ctypes.byref(msw), sp), P.handle)
        L.check(L.lib().tps_time_smoother(P.handle, lf, L.TPS_F32, 20, ctypes.byref(msw), sp), P.handle)
        sweep_ms = msw.value
        bytes_sweep, per_colour = smoother_bytes(dim, k, n, 4)
        colours = sum(1 for c in per_colour if c > 0)
        launch_ms = sweep_ms / colours
        launch_bytes = bytes_sweep / colours
        achieved = launch_bytes / (launch_ms * 1e-3) / 1e9

        # e2e through the public C API with host buffers (H2D b and x, D2H x)
        bh = b.cpu().pin_memory()
        xh = torch.zeros_like(bh).pin_memory()
        o = L.TpsSolveOpts(L.DRIVER_CG, L.VCYCLE_F32, 1, 100, 1e-10, 1e-300, 1)
        r = L.TpsReport()
        for _ in range(2):
            xh.zero_()
            L.check(L.lib().tps_solve_host(P.handle, ctypes.byref(o), bh.data_ptr(), xh.data_ptr(),
                                           ctypes.byref(r)), P.handle)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ne2e = max(3, args.steps // 2)
        for _ in range(ne2e):
            xh.zero_()
            L.check(L.lib().tps_solve_host(P.handle, ctypes.byref(o), bh.data_ptr(), xh.data_ptr(),
                                           ctypes.byref(r)), P.handle)
        torch.cuda.synchronize()
        e2e_ms = 1000 * (time.perf_counter() - t0) / ne2e

    t = torch.tensor([ms, ms64, e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, ms64, e2e_ms = t.tolist()
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    line = {
        "metric": METRIC, "value": world * nint / (ms * 1e-3), "unit": "DoF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 CG",
        "data": "synthetic (seeded sin-mode RHS per rank)",
        "config": {"workload": args.workload, "dim": dim, "degree": k, "cells": n,
                   "dofs": P.n_dofs(), "interior_dofs": nint, "levels": P.n_levels,
                   "rel_tol": 1e-10, "parallelism": f"replicas x{world}",
                   "l2": "vectors (136 MB FP64) larger than L2; no flush"},
        "iterations": rep.iterations, "final_rel_residual": resid_check,
        "fp64": {"ms_per_step": ms64, "value": world * nint / (ms64 * 1e-3),
                 "iterations": rep64.iterations},
        "mixed_speedup_vs_fp64": ms64 / ms,
        "error_vs_fp64_solve": err,
        "e2e": {"value": world * nint / (e2e_ms * 1e-3), "unit": "DoF/s",
                "h2d_bytes_per_step": 2 * 8 * P.n_dofs(), "d2h_bytes_per_step": 8 * P.n_dofs()},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": None,
                     "kernel": "smoother3d_kernel<4,float,TMA>",
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": launch_bytes, "launch_ms": launch_ms},
        "gpu_launches": args.steps * launches_per_solve(dim, P.n_levels, rep.iterations),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb, _ = cpu_baseline(args, dim, k, n, rep.iterations)
            line["cpu_baseline"] = cb
        except Exception as exc:  # report, never hide
            line["cpu_baseline"] = {"error": repr(exc)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
