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

At N = 1 the line also carries, measured after the headline's timed region,
a record of every other configuration under "configs": 2D Q2 64^2 (FP64 and
FP32 V-cycles), 3D Q7 32^3 (FP64, FP32 and TF32 tensor-core V-cycles), the
batched Q3 configuration (one graph launch per batch) and the adjoint check
of the variable-coefficient Q4 48^3 problem on 64 directions.  The CPU
baseline is one complete oracle solve of the headline instance.
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
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the sub-records of the other configurations (2D Q2 64^2, Q7 32^3, "
                         "batched Q3, adjoint Q4 48^3) that follow the headline measurement")
    ap.add_argument("--mode", default="solve",
                    choices=["solve", "smoother", "operator", "batch", "adjoint", "micro", "solves"],
                    help="smoother / operator: only time the finest-level smoother "
                         "sweeps / FP64 operator applications (small commands for kernel "
                         "profiling)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="--mode smoother: 3D smoother variant (0-2 CTA batches P, P/2, P/4; 3 one warp "
                         "per patch; -1 the library default)")
    ap.add_argument("--smoother", default="fp32", choices=["fp32", "tf32", "tf32x3", "fp64"],
                    help="--mode smoother: FP32 SIMT kernel, tensor-core kernel (TF32, or the "
                         "three-term TF32 split) or FP64")
    ap.add_argument("--directions", type=int, default=64,
                    help="--mode adjoint: random unit directions of the finite-difference check")
    ap.add_argument("--config", default=None,
                    help="JSON file of option values (keys as the long option names, '-' or '_'); "
                         "options given on the command line take precedence")
    args = ap.parse_args()
    if args.config:
        with open(args.config) as f:
            cfg = json.load(f)
        known = {a.dest for a in ap._actions}
        unknown = [key for key in cfg if key.replace("-", "_") not in known]
        if unknown:
            ap.error(f"unknown keys in {args.config}: {unknown}")
        ap.set_defaults(**{key.replace("-", "_"): v for key, v in cfg.items()})
        args = ap.parse_args()
    return args


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


def run_solves_once(args):
    """--mode solves: one FP32-V-cycle and one FP64-V-cycle solve of the
    workload after one warm-up solve of each (the small command for launch
    lists of whole solves); prints their iteration counts and times."""
    import torch
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    P = tps.PoissonProblem(dim, k, n)
    S = tps.MultigridSolvers(P)
    b = problems.make_rhs(args.workload)
    x = torch.zeros_like(b)
    out = {}
    for prec in ("fp32", "fp64", "fp32", "fp64"):
        x.zero_()
        _, rep = S.solve_cg(b, x, precision=prec, rel_tol=1e-10)
        torch.cuda.synchronize()
        out[prec] = {"iterations": rep.iterations, "ms": rep.time_ms}
    print(json.dumps({"mode": "solves", "workload": args.workload, **out}), flush=True)
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
    code = {"fp32": L.TPS_F32, "tf32": L.TPS_TF32, "tf32x3": L.TPS_TF32X3, "fp64": L.TPS_F64}[args.smoother]
    if args.variant >= 0 and args.smoother in ("fp32", "fp64"):
        P.set_smoother_variant(args.variant, args.smoother, lf)
    if args.warmup > 0:
        L.check(L.lib().tps_time_smoother(P.handle, lf, code, args.warmup, ctypes.byref(ms), sp), P.handle)
    L.check(L.lib().tps_time_smoother(P.handle, lf, code, max(args.steps, 1), ctypes.byref(ms), sp), P.handle)
    total, per = smoother_bytes(dim, k, n, 8 if args.smoother == "fp64" else 4)
    variant = P.smoother_variant(lf, args.smoother) if args.smoother in ("fp32", "fp64") else None
    print(json.dumps({"mode": "smoother", "smoother": args.smoother, "workload": args.workload,
                      "variant": variant, "ms_per_sweep": ms.value, "algorithmic_GBps": total / (ms.value * 1e-3) / 1e9}),
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
        self.first = threading.Event()
        self.mark = 0

    def start(self):
        """Starts nvidia-smi and returns once its first sample has arrived (at
        most 5 s), so that the samples cover the whole timed region that
        follows; only samples after this point are used."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.first.wait(5.0)
            self.mark = len(self.lines)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

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
        # the samples taken during the timed region (the last earlier one if none)
        lines = self.lines[self.mark:] or self.lines[-1:]
        for ln in lines:
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
    # q = A p and alpha: the operator, then the p.q dot and its finalize; in 3D
    # the operator forms the dot's partial sums itself (operator + finalize)
    q_alpha = 2 if dim == 3 else 3
    init = 1 + 1 + 2 + vcycle + 2 + q_alpha + 1 + 1
    per_it = vcycle + 2 + 1 + q_alpha + 1 + 1
    # one small copy kernel per host readback: the CG scalars after the set-up
    # and at each iteration's check, and the bounded-wait flag at the end
    readbacks = iterations + 2
    return init + per_it * max(iterations - 1, 0) + readbacks


def cg_iteration_bytes(dim: int, k: int, n_fine: int, n_levels: int, s: int) -> dict:
    """Algorithmic bytes of one MG-CG iteration (V-cycle in s-byte precision,
    FP64 outer CG), the sum the roofline of a whole solve is measured
    against.  Per level l >= 1 (N_l DoFs): two coloured sweeps (s (|U_c| +
    2 |I_c|) per colour), the residual s 3 N_l, the restriction s (N_l +
    N_l-1) and the prolongation-add s (2 N_l + N_l-1); the coarse level's
    single-patch solve is left out.  Outer CG on the fine level (N): q = A p
    8 2N; the beta dots r.z, q.z (z in the V-cycle precision) 16N + sN;
    p = z + beta p 16N + sN; x, r update and the V-cycle input 8 6N + sN."""
    n0 = n_fine >> (n_levels - 1)
    nd = [(n0 << l) * k + 1 for l in range(n_levels)]
    N = [v ** dim for v in nd]
    vc = 0
    for l in range(1, n_levels):
        vc += 2 * smoother_bytes(dim, k, n0 << l, s)[0]
        vc += s * 3 * N[l] + s * (N[l] + N[l - 1]) + s * (2 * N[l] + N[l - 1])
    nf = N[-1]
    cg = 8 * 2 * nf + (16 * nf + s * nf) + (16 * nf + s * nf) + (8 * 6 * nf + s * nf)
    return {"vcycle": vc, "outer_cg": cg, "total": vc + cg}


# DRAM traffic of the roofline kernel: ncu captures of its colour-0 launch
# (dram__bytes_read.sum + dram__bytes_write.sum, the launch's algorithmic
# bytes, the summary it comes from).  The bench reports it scaled to the
# average launch by algorithmic bytes; a kernel without a capture reports null.
TRAFFIC_CAPTURES = {
    ("smoother3d_warp_kernel<4,float>", "poisson3d_q4_64"):
        (136.6e6, 167.5e6, "profiles/smoother3d_warp_k4_f32_poisson3d_q4_64.md"),
    ("smoother3d_pair_kernel<4>", "poisson3d_q4_64"):
        (136.58e6, 167.5e6, "profiles/smoother3d_pair_k4_f32_poisson3d_q4_64.md"),
}


def traffic_per_launch(kernel: str, workload: str, launch_bytes: float):
    cap = TRAFFIC_CAPTURES.get((kernel, workload))
    return None if cap is None else cap[0] * launch_bytes / cap[1]


def workload_config(args, world: int) -> dict:
    """The workload description shared by both arms' JSON lines."""
    from gputensorproductsmoother_b200 import problems, split_cells
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    _, levels = split_cells(n)
    return {"workload": args.workload, "dim": dim, "degree": k, "cells": n,
            "dofs": (n * k + 1) ** dim, "interior_dofs": problems.interior_dofs(dim, k, n),
            "levels": levels, "rel_tol": 1e-10, "parallelism": f"replicas x{world}",
            "l2": "vectors (136 MB FP64) larger than L2; no flush"}


def oracle_solve_timed(args, seed: int = 0):
    """One full solve of the workload by the CPU oracle (the same algorithm:
    coloured vertex-patch smoother, FP32 V-cycle, FP64 flexible CG to a 1e-10
    relative residual, from x = 0) on all host cores; returns (seconds,
    iterations, final relative residual)."""
    from oracle import oracle as O
    from gputensorproductsmoother_b200 import problems, split_cells
    dim, k, n, gen = problems.WORKLOADS[args.workload]
    nc, nl = split_cells(n)
    b = gen(dim, k, n, seed, "cpu").numpy()
    H = O.Hierarchy(dim, k, nc, nl)
    t0 = time.perf_counter()
    _, it, hist = H.solve_cg(b, precision=1, symmetric=True, rel_tol=1e-10)
    t = time.perf_counter() - t0
    return t, it, float(hist[-1] / hist[0])


def host_threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def cpu_baseline(args):
    """The CPU oracle timed on the host cores: one complete solve of the same
    instance (measured, not scaled)."""
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    t, it, res = oracle_solve_timed(args)
    nint = problems.interior_dofs(dim, k, n)
    return {"value": nint / t, "unit": "DoF/s", "cores": host_threads(), "kind": "port",
            "sample": f"one complete solve of the same {n}^{dim} Q{k} instance ({it} CG iterations to "
                      f"{res:.1e}, {t:.1f} s, measured)"}


def run_reference(args):
    """Reference arm: the reference's implementation of this path needs a GPU
    and deal.II, so its CPU-runnable counterpart is the oracle port (the same
    algorithm).  Each step is one complete solve of the workload on all host
    cores, timed; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    nint = problems.interior_dofs(dim, k, n)
    times, its = [], None
    for s in range(args.warmup + args.steps):
        t, it, res = oracle_solve_timed(args)
        if s >= args.warmup:
            times.append(t)
            its = it
    ms = 1000 * statistics.mean(times)
    val = nint / (ms / 1000)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "DoF/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 CG",
            "data": "synthetic (seeded sin-mode RHS)", "config": workload_config(args, world),
            "iterations": its, "final_rel_residual": res,
            "cpu_baseline": {"value": val, "unit": "DoF/s", "cores": host_threads(), "kind": "port",
                             "sample": f"each step one complete solve of the {n}^{dim} Q{k} instance "
                                       f"({its} CG iterations, measured)"},
            "e2e": {"value": val, "unit": "DoF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_micro(args):
    """Micro-benchmarks of the level operations (the reference's
    apps/benchmark_mg.cu:238-503): operator FP64/FP32, transfers FP64/FP32
    between the two finest levels, and the finest-level smoother for every
    compiled patches-per-block variant (FP64, FP32) and the tensor-core
    variant.  Best of 5 repetitions of 10 calls, CUDA events; one JSON line."""
    import torch
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import _lib as L
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[args.workload]
    P = tps.PoissonProblem(dim, k, n)
    lf = P.n_levels - 1
    N, Nc = P.n_dofs(lf), P.n_dofs(lf - 1)
    rows = []

    def best(fn, calls=10, reps=5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fn()
        t = 1e30
        for _ in range(reps):
            e0.record()
            for _ in range(calls):
                fn()
            e1.record()
            torch.cuda.synchronize()
            t = min(t, e0.elapsed_time(e1) / calls)
        return t

    for dt, name in ((torch.float64, "DP"), (torch.float32, "SP")):
        src = problems.make_rhs(args.workload).to(dt)
        dst = torch.empty_like(src)
        A = tps.LaplaceOperator(P)
        ms = best(lambda: A.vmult(dst, src))
        rows.append({"name": f"Mat-vec {name}", "ms": ms, "dof_per_s": N / (ms * 1e-3),
                     "GBps": 2 * src.element_size() * N / (ms * 1e-3) / 1e9})
        T = tps.MGTransferCUDA(P)
        fine = torch.ones(N, dtype=dt, device="cuda")
        coarse = torch.ones(Nc, dtype=dt, device="cuda")
        ms = best(lambda: T.prolongate_and_add(lf, fine, coarse))
        rows.append({"name": f"Prolongation {name}", "ms": ms, "dof_per_s": N / (ms * 1e-3)})
        ms = best(lambda: T.restrict_and_add(lf, coarse, fine))
        rows.append({"name": f"Restriction {name}", "ms": ms, "dof_per_s": N / (ms * 1e-3)})
    for dtname, code in (("DP", L.TPS_F64), ("SP", L.TPS_F32)):
        ppb = (ctypes.c_int * L.SMOOTHER_VARIANTS)()
        L.check(L.lib().tps_smoother_variants(P.handle, code, ppb), P.handle)
        seen = set()
        for v in range(L.SMOOTHER_VARIANTS):
            if ppb[v] in seen:
                continue
            seen.add(ppb[v])
            L.check(L.lib().tps_set_smoother_variant(P.handle, code, lf, v), P.handle)
            P.time_smoother(dtype="fp64" if code == L.TPS_F64 else "fp32", sweeps=2)
            ms = P.time_smoother(dtype="fp64" if code == L.TPS_F64 else "fp32", sweeps=10)
            total, _ = smoother_bytes(dim, k, n, 8 if code == L.TPS_F64 else 4)
            label = {-1: "warp/patch", -2: "2 patches/warp f32x2"}.get(ppb[v], f"ppb={ppb[v]}")
            rows.append({"name": f"Smooth {dtname} {label}", "ms": ms, "dof_per_s": N / (ms * 1e-3),
                         "GBps": total / (ms * 1e-3) / 1e9})
        L.check(L.lib().tps_set_smoother_variant(P.handle, code, lf, 0), P.handle)
    if dim == 3 and k >= 2:
        P.time_smoother(dtype="tf32", sweeps=2)
        ms = P.time_smoother(dtype="tf32", sweeps=10)
        total, _ = smoother_bytes(dim, k, n, 4)
        rows.append({"name": "Smooth TF32 tensor cores", "ms": ms, "dof_per_s": N / (ms * 1e-3),
                     "GBps": total / (ms * 1e-3) / 1e9})
    print(json.dumps({"mode": "micro", "workload": args.workload, "dofs": N, "rows": rows}), flush=True)
    P.close()


def max_over_ranks(values, world: int, device: str = "cuda"):
    """Element-wise maximum of per-rank timings over the process group (the
    whole job is as slow as its slowest rank); identity for one rank."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_throughput(world: int, units_per_rank: float, ms: float) -> float:
    """Whole-job units per second: every rank solves its own instance of
    `units_per_rank` units, the job takes the slowest rank's `ms`."""
    return world * units_per_rank / (ms * 1e-3)


def batch_systems(seed: int = 0):
    """Batched workload: 32 right-hand sides on one 32^3 Q3 mesh plus 12
    independent Q3 meshes with 8..48 cells per direction drawn from the seed
    (sizes n_c 2^l with n_c in {2, 3, 5}, so the coarse level stays a single
    patch or a small dense solve)."""
    import numpy as np
    sizes = [n for n in range(8, 49) if any(n % c == 0 and ((n // c) & (n // c - 1)) == 0 for c in (2, 3, 5))]
    rng = np.random.default_rng(seed)
    meshes = sorted(int(v) for v in rng.choice(sizes, 12, replace=True))
    return [(3, 3, 32)] * 32 + [(3, 3, n) for n in meshes]


def run_batch(args):
    """--mode batch: prints measure_batch's record as one JSON line."""
    print(json.dumps(dict(mode="batch", **measure_batch(args.warmup, args.steps))), flush=True)


def measure_batch(warmup: int, steps: int) -> dict:
    """Times `steps` batched solves (one graph launch each) of batch_systems()
    after `warmup`: FP32 V-cycle, FP64 CG to 1e-10, right-hand sides i.i.d.
    uniform[-1,1] nodal values."""
    import numpy as np
    import torch
    import gputensorproductsmoother_b200 as tps
    systems = batch_systems()
    B = tps.BatchSolver(systems)
    rng = np.random.default_rng(1)
    rhs = []
    for (d, k, n) in systems:
        N1 = n * k + 1
        v = rng.uniform(-1, 1, N1 ** d)
        idx = np.stack(np.unravel_index(np.arange(N1 ** d), (N1,) * d))
        v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
        rhs.append(torch.tensor(v, device="cuda"))
    xs = [torch.zeros_like(b) for b in rhs]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for _ in range(max(warmup, 1)):
            for x in xs:
                x.zero_()
            _, reps = B.solve(rhs, xs, precision="fp32", rel_tol=1e-10)
        times = []
        for _ in range(max(steps, 1)):
            for x in xs:
                x.zero_()
            _, reps = B.solve(rhs, xs, precision="fp32", rel_tol=1e-10)
            times.append(reps[0].time_ms)
    torch.cuda.synchronize()
    nint = sum((n * k - 1) ** d for (d, k, n) in systems)
    ms = statistics.median(times)
    B.close()
    return {"metric": "batched MG-CG DoF/s to 1e-10 (one graph launch per batch)",
            "value": nint / (ms * 1e-3), "unit": "DoF/s", "ms_per_batch": ms, "steps": steps,
            "systems": len(systems), "meshes": sorted({n for (_, _, n) in systems}),
            "interior_dofs": nint, "iterations": sorted({r.iterations for r in reps}),
            "all_converged": all(r.converged for r in reps),
            "max_final_residual": max(r.final_residual for r in reps),
            "graph_launches_per_batch": 1}


def run_adjoint(args):
    """--mode adjoint: prints measure_adjoint's record as one JSON line."""
    print(json.dumps(dict(mode="adjoint", **measure_adjoint(args.directions))), flush=True)


def measure_adjoint(directions: int) -> dict:
    """Adjoint check of -div(kappa grad u) = f, Q4, 48^3 cells (coarse 3^3),
    kappa = exp(N(0, 0.5^2)) per cell, J = 0.5 ||u - u_t||^2 with u_t a smooth
    field of 8 random sine modes: dJ/df and dJ/dkappa (FP64, adjoint solve)
    against central differences (h = 1e-6) on --directions random directions
    (i.i.d. N(0,1) entries for f, relative N(0,1) perturbations kappa * N(0,1)
    for kappa; unit-norm directions over 7.2M DoFs would leave a directional
    derivative ~1/2700 of the gradient norm, below the rounding of J / h).
    Returns the worst and median relative deviations."""
    import numpy as np
    import torch
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import problems
    dim, k, n = 3, 4, 48
    rng = np.random.default_rng(0)
    kap = torch.tensor(np.exp(rng.normal(0.0, 0.5, n ** dim)), device="cuda")
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    N = P.n_dofs()
    f = torch.tensor(rng.uniform(-1, 1, N), device="cuda")
    with torch.no_grad():
        u0 = tps.autograd.solve(P, f, kap, rel_tol=1e-13)
    ut = problems.sine_modes_rhs(dim, k, n, 5, 8, "cuda")
    ut = ut * (u0.abs().max() / ut.abs().max())

    def J(f_, k_):
        u = tps.autograd.solve(P, f_, k_, rel_tol=1e-13)
        return 0.5 * ((u - ut) ** 2).sum()

    fv, kv = f.clone().requires_grad_(True), kap.clone().requires_grad_(True)
    t0 = time.perf_counter()
    j = J(fv, kv)
    j.backward()
    t_grad = time.perf_counter() - t0
    gf, gk = fv.grad.detach(), kv.grad.detach()
    h = 1e-6
    worst_f = worst_k = 0.0
    devs_f, devs_k = [], []
    t0 = time.perf_counter()
    for d in range(directions):
        df = torch.tensor(rng.standard_normal(N), device="cuda")
        dk = torch.tensor(rng.standard_normal(n ** dim), device="cuda") * kap
        with torch.no_grad():
            fd_f = (J(f + h * df, kap) - J(f - h * df, kap)) / (2 * h)
            fd_k = (J(f, kap + h * dk) - J(f, kap - h * dk)) / (2 * h)
        devs_f.append(abs((gf * df).sum().item() - fd_f.item()) / abs(fd_f.item()))
        devs_k.append(abs((gk * dk).sum().item() - fd_k.item()) / abs(fd_k.item()))
        worst_f, worst_k = max(devs_f), max(devs_k)
    t_fd = time.perf_counter() - t0
    P.close()
    return {"workload": "kappa_q4_48", "dofs": N, "directions": directions,
            "fd_step": h, "max_rel_dev_df": worst_f, "max_rel_dev_dkappa": worst_k,
            "median_rel_dev_df": statistics.median(devs_f), "median_rel_dev_dkappa": statistics.median(devs_k),
            "within_1e-6": worst_f <= 1e-6 and worst_k <= 1e-6,
            "s_forward_plus_adjoint": t_grad, "s_finite_differences": t_fd}


def measure_solves(workload: str, precisions, warmup: int = 1, reps: int = 3) -> dict:
    """Solves of one configuration from x = 0 to 1e-10 with each V-cycle
    precision (the first must be "fp64": the FP64 GPU solution the others'
    errors refer to): best time of `reps` (CUDA events on the solving
    stream), iterations, final residual, DoF/s.  With both "fp32" and "tf32":
    whether the TF32 V-cycle used the tensor cores on any level, and at
    degrees 5..7 the finest level's sweep time on the FP32 SIMT and the
    tensor-core (TF32) smoothers."""
    import torch
    import gputensorproductsmoother_b200 as tps
    from gputensorproductsmoother_b200 import problems
    dim, k, n, _ = problems.WORKLOADS[workload]
    P = tps.PoissonProblem(dim, k, n)
    S = tps.MultigridSolvers(P)
    b = problems.make_rhs(workload)
    x = torch.zeros_like(b)
    nint = problems.interior_dofs(dim, k, n)
    out = {"dofs": P.n_dofs(), "interior_dofs": nint}
    stream = torch.cuda.Stream()
    x64 = None
    histories = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for prec in precisions:
            for _ in range(max(warmup, 1)):
                x.zero_()
                _, rep = S.solve_cg(b, x, precision=prec, rel_tol=1e-10)
            best = 1e30
            for _ in range(max(reps, 1)):
                x.zero_()
                e0.record(stream)
                _, rep = S.solve_cg(b, x, precision=prec, rel_tol=1e-10)
                e1.record(stream)
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            rec = {"ms": best, "dof_per_s": nint / (best * 1e-3), "iterations": rep.iterations,
                   "final_rel_residual": rep.final_residual}
            if x64 is None:
                x64 = x.clone()
            else:
                rec["error_vs_fp64_solve"] = (torch.linalg.norm(x - x64) / torch.linalg.norm(x64)).item()
            histories[prec] = list(rep.history)
            out[prec] = rec
    if "fp64" in out:
        for prec in precisions[1:]:
            out[prec]["speedup_vs_fp64"] = out["fp64"]["ms"] / out[prec]["ms"]
    if "tf32" in out and "fp32" in out:
        # the TF32 V-cycle runs the tensor-core smoother only on the levels
        # where it is faster; a residual history identical to the FP32
        # V-cycle's shows that it ran on none
        out["tf32"]["tensor_core_levels_used"] = histories["tf32"] != histories["fp32"]
        if dim == 3 and k >= 5:
            lf = P.n_levels - 1
            sweep = {}
            for d in ("fp32", "tf32"):
                P.time_smoother(lf, d, 2)
                sweep[d] = min(P.time_smoother(lf, d, 10) for _ in range(3))
            out["finest_level_sweep_ms"] = {"fp32_simt": sweep["fp32"], "tf32_tensor_cores": sweep["tf32"],
                                            "kernel": f"smoother3d_tc_kernel<{k}>"}
    P.close()
    return out


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
    if args.mode == "solves":
        run_solves_once(args)
        return
    if args.mode == "batch":
        run_batch(args)
        return
    if args.mode == "micro":
        run_micro(args)
        return
    if args.mode == "adjoint":
        run_adjoint(args)
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

        # the same FP64 CG with the TF32 V-cycle (3D degrees 2..4: the
        # tensor-core patch-GEMM smoother), reported beside the headline
        tf32 = None
        if dim == 3 and k >= 2:
            for _ in range(max(1, args.warmup // 2)):
                reptc = solve("tf32")
            e0.record(stream)
            for _ in range(n64):
                reptc = solve("tf32")
            e1.record(stream)
            torch.cuda.synchronize()
            mstc = e0.elapsed_time(e1) / n64
            errtc = (torch.linalg.norm(x - x64) / torch.linalg.norm(x64)).item()
            tf32 = {"ms_per_step": mstc, "value": job_throughput(world, nint, mstc), "iterations": reptc.iterations,
                    "final_rel_residual": reptc.final_residual, "error_vs_fp64_solve": errtc,
                    "speedup_vs_fp64": ms64 / mstc}

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
        kernel_name = {3: f"smoother3d_warp_kernel<{k},float>", 4: f"smoother3d_pair_kernel<{k}>"}.get(
            P.smoother_variant(lf, "fp32"), f"smoother3d_kernel<{k},float,TMA>")
        bytes_sweep, per_colour = smoother_bytes(dim, k, n, 4)
        colours = sum(1 for c in per_colour if c > 0)
        launch_ms = sweep_ms / colours
        launch_bytes = bytes_sweep / colours
        achieved = launch_bytes / (launch_ms * 1e-3) / 1e9
        # the same sweep with the TF32 patch-GEMM smoother (tensor cores)
        tf32_sweep_ms = None
        if tf32 is not None:
            L.check(L.lib().tps_time_smoother(P.handle, lf, L.TPS_TF32, 3, ctypes.byref(msw), sp), P.handle)
            L.check(L.lib().tps_time_smoother(P.handle, lf, L.TPS_TF32, 20, ctypes.byref(msw), sp), P.handle)
            tf32_sweep_ms = msw.value

        # e2e through the public C API with host buffers: H2D of b (pinned), the
        # solve from x = 0 (the reference's starting guess, set on the device),
        # D2H of x
        bh = b.cpu().pin_memory()
        xh = torch.empty_like(bh).pin_memory()
        o = L.TpsSolveOpts(L.DRIVER_CG, L.VCYCLE_F32, 1, 100, 1e-10, 1e-300, 1)
        r = L.TpsReport()
        for _ in range(2):
            L.check(L.lib().tps_solve_host_guess(P.handle, ctypes.byref(o), bh.data_ptr(), None, xh.data_ptr(),
                                                 ctypes.byref(r)), P.handle)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ne2e = max(3, args.steps // 2)
        for _ in range(ne2e):
            L.check(L.lib().tps_solve_host_guess(P.handle, ctypes.byref(o), bh.data_ptr(), None, xh.data_ptr(),
                                                 ctypes.byref(r)), P.handle)
        torch.cuda.synchronize()
        e2e_serial_ms = 1000 * (time.perf_counter() - t0) / ne2e
        # the same steps as one sequence (tps_solve_host_many): each step still
        # copies its b in and its x out, overlapped with the neighbouring solves
        # (b[i+1] in and x[i-1] out while solve i runs); outputs alternate
        # between two pinned buffers
        xh2 = torch.empty_like(bh).pin_memory()
        nseq = max(4, args.steps)
        bp = (ctypes.c_void_p * nseq)(*([bh.data_ptr()] * nseq))
        xp = (ctypes.c_void_p * nseq)(*[(xh if i % 2 == 0 else xh2).data_ptr() for i in range(nseq)])
        reps = (L.TpsReport * nseq)()
        L.check(L.lib().tps_solve_host_many(P.handle, ctypes.byref(o), 2, bp, xp, reps), P.handle)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L.check(L.lib().tps_solve_host_many(P.handle, ctypes.byref(o), nseq, bp, xp, reps), P.handle)
        torch.cuda.synchronize()
        e2e_ms = 1000 * (time.perf_counter() - t0) / nseq
        e2e_err = max((torch.linalg.norm(v.to(x.device) - x64) / torch.linalg.norm(x64)).item() for v in (xh, xh2))

    ms, ms64, e2e_ms, e2e_serial_ms = max_over_ranks([ms, ms64, e2e_ms, e2e_serial_ms], world)
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    line = {
        "metric": METRIC, "value": job_throughput(world, nint, ms), "unit": "DoF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 V-cycle / f64 CG",
        "data": "synthetic (seeded sin-mode RHS per rank)",
        "config": workload_config(args, world),
        "iterations": rep.iterations, "final_rel_residual": resid_check,
        "fp64": {"ms_per_step": ms64, "value": job_throughput(world, nint, ms64),
                 "iterations": rep64.iterations},
        "mixed_speedup_vs_fp64": ms64 / ms,
        "tf32_vcycle": tf32,
        "tf32_smoother": None if tf32_sweep_ms is None else {
            "kernel": f"smoother3d_gemm_kernel<{k}>", "ms_per_sweep": tf32_sweep_ms,
            "achieved_GBps": bytes_sweep / (tf32_sweep_ms * 1e-3) / 1e9,
            "frac": bytes_sweep / (tf32_sweep_ms * 1e-3) / 1e9 / hbm_peak},
        "error_vs_fp64_solve": err,
        "e2e": {"value": job_throughput(world, nint, e2e_ms), "unit": "DoF/s",
                "h2d_bytes_per_step": 8 * P.n_dofs(), "d2h_bytes_per_step": 8 * P.n_dofs(),
                "steps": nseq, "api": "tps_solve_host_many (copies overlapped with the neighbouring solves)",
                "serial_value": job_throughput(world, nint, e2e_serial_ms),
                "serial_api": "tps_solve_host_guess per step (copies not overlapped)",
                "error_vs_fp64_solve": e2e_err},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak,
                     "traffic": traffic_per_launch(kernel_name, args.workload, launch_bytes),
                     "traffic_unit": "bytes per launch",
                     "traffic_source": TRAFFIC_CAPTURES.get((kernel_name, args.workload), (0, 0, None))[2],
                     "kernel": kernel_name,
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": launch_bytes, "launch_ms": launch_ms},
        "gpu_launches": args.steps * launches_per_solve(dim, P.n_levels, rep.iterations),
        "clocks": clocks,
    }
    # the whole solve against HBM: algorithmic bytes of its CG iterations (the
    # initial residual and the convergence checks left out) / the solve time
    itb = cg_iteration_bytes(dim, k, n, P.n_levels, 4)
    solve_gbps = itb["total"] * rep.iterations / (ms * 1e-3) / 1e9
    line["solve_roofline"] = {"bytes_per_iteration": itb, "iterations": rep.iterations,
                              "achieved": solve_gbps, "peak": hbm_peak, "unit": "GB/s",
                              "frac": solve_gbps / hbm_peak,
                              "model": "sum over levels of 2 sweeps, residual, restriction, "
                                       "prolongation + outer-CG vector and operator traffic, "
                                       "per iteration x iterations / solve time"}
    if rank == 0 and world == 1 and not args.no_configs:
        # every other configuration, measured after the headline's timed region
        subs = {}
        for name, fn in (("poisson2d_q2_64", lambda: measure_solves("poisson2d_q2_64", ("fp64", "fp32"))),
                         ("poisson3d_q7_32", lambda: measure_solves("poisson3d_q7_32", ("fp64", "fp32", "tf32"))),
                         ("batched_q3_32rhs_12meshes", lambda: measure_batch(2, 5)),
                         ("adjoint_kappa_q4_48", lambda: measure_adjoint(64))):
            try:
                subs[name] = fn()
            except Exception as exc:  # report, never hide
                subs[name] = {"error": repr(exc)}
        line["configs"] = subs
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(args)
        except Exception as exc:  # report, never hide
            line["cpu_baseline"] = {"error": repr(exc)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
