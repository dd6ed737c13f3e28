"""The benchmark configurations at their full sizes (1 GPU): each solve
converges to its tolerance and agrees with the FP64 solve (or the CPU oracle
where that is quick).  Seeded synthetic inputs with the configurations'
shapes and distributions."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import problems

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return (a - b).abs().max().item() / b.abs().max().item()


def test_config_2d_q2_64(cuda, oracle):
    """2D Q2 on 64^2 cells, f i.i.d. U[-1,1] nodal values, b = M f, FP64,
    CG to 1e-10: identical iteration count and solution as the oracle."""
    b = problems.make_rhs("poisson2d_q2_64")
    P = tps.PoissonProblem(2, 2, 64)
    x, rep = tps.MultigridSolvers(P).solve_cg(b, precision="fp64", rel_tol=1e-10)
    H = oracle.Hierarchy(2, 2, P.n_coarse, P.n_levels)
    xr, itr, _ = H.solve_cg(b.cpu().numpy(), precision=0, symmetric=True, rel_tol=1e-10)
    assert rep.converged and rep.iterations == itr
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xr) <= 1e-12 * np.linalg.norm(xr)
    assert np.abs(xg - xr).max() <= 1e-11 * np.abs(xr).max()


def test_config_3d_q4_64_mixed_vs_fp64(cuda):
    """3D Q4 on 64^3 cells, 8 seeded sine modes: FP32 and FP64 V-cycles under
    the FP64 CG reach 1e-10 and the same solution."""
    b = problems.make_rhs("poisson3d_q4_64")
    P = tps.PoissonProblem(3, 4, 64)
    MG = tps.MultigridSolvers(P)
    x64, r64 = MG.solve_cg(b, precision="fp64", rel_tol=1e-10)
    x32, r32 = MG.solve_cg(b, precision="fp32", rel_tol=1e-10)
    assert r64.converged and r32.converged and r32.final_residual <= 1e-10
    assert relerr(x32, x64) < 1e-8


def test_config_3d_q7_32(cuda):
    """3D Q7 on 32^3 cells, f i.i.d. N(0,1) nodal values: FP32 SIMT and TF32
    tensor-core V-cycles under the FP64 CG reach 1e-10, agree with FP64."""
    b = problems.make_rhs("poisson3d_q7_32")
    P = tps.PoissonProblem(3, 7, 32)
    MG = tps.MultigridSolvers(P)
    x64, r64 = MG.solve_cg(b, precision="fp64", rel_tol=1e-10)
    for prec in ("fp32", "tf32"):
        x, r = MG.solve_cg(b, precision=prec, rel_tol=1e-10)
        assert r.converged and r.final_residual <= 1e-10
        assert relerr(x, x64) < 1e-8
        assert r.iterations <= r64.iterations + 2


def test_config_batched(cuda):
    """32 right-hand sides on 32^3 Q3 plus 12 Q3 meshes of 8^3..48^3 in one
    graph launch: every system reaches 1e-10 and matches its single solve."""
    import bench
    systems = bench.batch_systems()
    B = tps.BatchSolver(systems)
    rng = np.random.default_rng(1)
    rhs = []
    for (d, k, n) in systems:
        N1 = n * k + 1
        v = rng.uniform(-1, 1, N1 ** d)
        idx = np.stack(np.unravel_index(np.arange(N1 ** d), (N1,) * d))
        v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
        rhs.append(torch.tensor(v, device="cuda"))
    xs, reps = B.solve(rhs, precision="fp32", rel_tol=1e-10)
    assert all(r.converged and r.final_residual <= 1e-10 for r in reps)
    for i in (0, 31, 32, 43):  # one of the RHS block and the smallest / largest meshes
        d, k, n = systems[i]
        P = tps.PoissonProblem(d, k, n)
        x1, r1 = tps.MultigridSolvers(P).solve_cg(rhs[i], precision="fp32", rel_tol=1e-10)
        assert reps[i].iterations == r1.iterations and relerr(xs[i], x1) < 1e-12
        P.close()
    B.close()
