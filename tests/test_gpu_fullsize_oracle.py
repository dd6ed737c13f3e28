"""The benchmark configurations at their FULL sizes against the CPU oracle.

Each GPU solve runs through the C ABI (libtps.so); the oracle (oracle/, C,
OpenMP) solves the same seeded instance on the host with the same algorithm.
The tolerance is the one the plain FP64 path must meet against the reference
implementation: identical CG iteration counts and a solution within 1e-12
relative (2-norm).  The mixed solves (FP32 SIMT or TF32 tensor-core V-cycle
under the FP64 CG) state their error against the oracle's FP64 solve.

Each oracle solve of a 3D configuration takes tens of seconds on the host
cores, so the FP64 oracle solution of a configuration is computed once and
shared by the tests of that configuration.
"""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import problems

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12  # FP64 GPU solve vs FP64 oracle solve (relative 2-norm)
TOL_MIXED = 1e-8  # mixed-precision V-cycle solve vs FP64 oracle solve (both to 1e-10 residual)

_ORACLE_CACHE = {}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _oracle_solution(oracle, key, dim, k, n, b, precision=0):
    """FP64-CG solution of the oracle (V-cycle in FP64 for precision 0, FP32
    for 1) to 1e-10, computed once per (key, precision)."""
    ck = (key, precision)
    if ck not in _ORACLE_CACHE:
        nc, nl = tps.split_cells(n)
        H = oracle.Hierarchy(dim, k, nc, nl)
        x, it, hist = H.solve_cg(b, precision=precision, symmetric=True, rel_tol=1e-10)
        _ORACLE_CACHE[ck] = (H, x, it, hist)
    return _ORACLE_CACHE[ck]


@pytest.mark.parametrize("workload", ["poisson3d_q4_64", "poisson3d_q7_32"])
def test_fullsize_fp64_matches_oracle(cuda, oracle, workload):
    """Plain FP64 path at full size: identical iteration count, solution within
    1e-12 of the oracle's, residual histories equal to 1e-6 relative."""
    dim, k, n, _ = problems.WORKLOADS[workload]
    b = problems.make_rhs(workload, device="cpu").numpy()
    H, xr, itr, histr = _oracle_solution(oracle, workload, dim, k, n, b)
    P = tps.PoissonProblem(dim, k, n)
    x, rep = tps.MultigridSolvers(P).solve_cg(torch.tensor(b, device="cuda"), precision="fp64",
                                              rel_tol=1e-10)
    assert rep.converged and rep.iterations == itr, (rep.iterations, itr)
    err = _rel(x.cpu().numpy(), xr)
    assert err <= TOL_FP64, err
    np.testing.assert_allclose(rep.history, histr, rtol=1e-6)
    P.close()


@pytest.mark.parametrize("workload,precisions", [("poisson3d_q4_64", ("fp32", "tf32", "tf32x3")),
                                                 ("poisson3d_q7_32", ("fp32", "tf32"))])
def test_fullsize_mixed_error_vs_oracle(cuda, oracle, workload, precisions):
    """Mixed-precision V-cycles at full size: converged to 1e-10 (true residual
    computed by the oracle) and within 1e-8 of the oracle's FP64 solve; the
    FP32 V-cycle takes the oracle's FP32-V-cycle iteration count."""
    dim, k, n, _ = problems.WORKLOADS[workload]
    b = problems.make_rhs(workload, device="cpu").numpy()
    H, xr, _, _ = _oracle_solution(oracle, workload, dim, k, n, b)
    _, _, it32, _ = _oracle_solution(oracle, workload, dim, k, n, b, precision=1)
    P = tps.PoissonProblem(dim, k, n)
    MG = tps.MultigridSolvers(P)
    bd = torch.tensor(b, device="cuda")
    for prec in precisions:
        x, rep = MG.solve_cg(bd, precision=prec, rel_tol=1e-10)
        xh = x.cpu().numpy()
        assert rep.converged, prec
        r = b - H.vmult(xh)
        assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b), prec
        err = _rel(xh, xr)
        assert err <= TOL_MIXED, (prec, err)
        if prec in ("fp32", "tf32x3"):  # FP32-accurate V-cycles: the oracle's FP32 count
            assert rep.iterations == it32, (prec, rep.iterations, it32)
    P.close()


def test_config_2d_q2_64_fp64_matches_oracle(cuda, oracle):
    """2D Q2 64^2 (f i.i.d. U[-1,1] nodal, b = M f): FP64 CG to 1e-10 with the
    oracle's iteration count and solution within 1e-12."""
    b = problems.make_rhs("poisson2d_q2_64", device="cpu").numpy()
    H, xr, itr, _ = _oracle_solution(oracle, "poisson2d_q2_64", 2, 2, 64, b)
    P = tps.PoissonProblem(2, 2, 64)
    x, rep = tps.MultigridSolvers(P).solve_cg(torch.tensor(b, device="cuda"), precision="fp64",
                                              rel_tol=1e-10)
    assert rep.converged and rep.iterations == itr
    assert _rel(x.cpu().numpy(), xr) <= TOL_FP64
    P.close()


def _batch_rhs(systems):
    rng = np.random.default_rng(1)
    rhs = []
    for (d, k, n) in systems:
        N1 = n * k + 1
        v = rng.uniform(-1, 1, N1 ** d)
        idx = np.stack(np.unravel_index(np.arange(N1 ** d), (N1,) * d))
        v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
        rhs.append(v)
    return rhs


def test_batched_systems_match_oracle(cuda, oracle):
    """The batched configuration (32 RHS on 32^3 Q3 + 12 Q3 meshes in one
    graph launch): with the FP64 V-cycle three systems (a right-hand side of
    the shared mesh, the smallest and the largest mesh) take the oracle's
    iteration counts and match its solutions to 1e-12; with the FP32 V-cycle
    they are within 1e-8 of the oracle's FP64 solutions."""
    import bench
    systems = bench.batch_systems()
    rhs = _batch_rhs(systems)
    B = tps.BatchSolver(systems)
    dev = [torch.tensor(v, device="cuda") for v in rhs]
    x64, reps64 = B.solve(dev, precision="fp64", rel_tol=1e-10)
    x32, reps32 = B.solve(dev, precision="fp32", rel_tol=1e-10)
    picks = [0, 32, len(systems) - 1]
    for i in picks:
        d, k, n = systems[i]
        _, xr, itr, _ = _oracle_solution(oracle, ("batch", i), d, k, n, rhs[i])
        assert reps64[i].converged and reps64[i].iterations == itr, (i, reps64[i].iterations, itr)
        assert _rel(x64[i].cpu().numpy(), xr) <= TOL_FP64, i
        assert reps32[i].converged
        assert _rel(x32[i].cpu().numpy(), xr) <= TOL_MIXED, i
    B.close()
