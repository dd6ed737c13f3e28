"""GPU tests of the additive vertex-patch Schwarz step (no reference
counterpart: the reference's sweep is the coloured multiplicative one; the 2D
benchmark configuration names the additive form): one step and the V-cycle
with additive smoothing against the oracle's restatement, and the 2D Q2 64^2
configuration solved with it."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def interior_random(dim, N1, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, N1 ** dim)
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return v


@pytest.mark.parametrize("dim,k,n", [(2, 1, 8), (2, 2, 8), (2, 3, 4), (2, 4, 8), (3, 1, 4), (3, 2, 4), (3, 3, 4),
                                     (3, 4, 4), (3, 4, 8)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("zero_init", [False, True])
def test_additive_step_matches_oracle(cuda, oracle, dim, k, n, dtype, zero_init):
    P = tps.PoissonProblem(dim, k, n)
    N = P.n_dofs()
    rng = np.random.default_rng(500 + 10 * dim + k)
    x0, b = rng.uniform(-1, 1, N), rng.uniform(-1, 1, N)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    omega = 1.0 / 2 ** dim  # the default damping
    ref = oracle.smoother_additive(dim, k, n, x0.astype(npdt), b.astype(npdt), omega, zero_init=zero_init)
    x = torch.tensor(x0, dtype=dtype, device="cuda")
    sm = tps.PatchSmoother(P, variant="additive")
    (sm.vmult if zero_init else sm.step)(x, torch.tensor(b, dtype=dtype, device="cuda"))
    torch.cuda.synchronize()
    assert relerr(x.cpu().numpy(), ref) < (TOL64 if dtype == torch.float64 else TOL32)
    P.close()


@pytest.mark.parametrize("dim,k,n", [(2, 2, 16), (3, 2, 8), (3, 4, 8)])
@pytest.mark.parametrize("precision,oprec,tol", [("fp64", 0, TOL64), ("fp32", 1, 1e-4)])
def test_additive_vcycle_matches_oracle(cuda, oracle, dim, k, n, precision, oprec, tol):
    P = tps.PoissonProblem(dim, k, n)
    omega = 0.8 / 2 ** dim
    P.set_smoother_kind("additive", omega)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    H.set_additive(omega)
    src = np.random.default_rng(600 + k).uniform(-1, 1, P.n_dofs())
    ref = H.vcycle(src, precision=oprec)
    dst = P.new_vector()
    tps.MultigridSolvers(P).vmult(dst, torch.tensor(src, device="cuda"), precision=precision)
    torch.cuda.synchronize()
    assert relerr(dst.cpu().numpy(), ref) < tol
    P.close()


def test_additive_cg_2d_q2_64(cuda, oracle):
    """2D Q2, 64^2 cells, coarse 2x2 cells, 1 pre / 1 post additive step
    (damping 1/4), CG to 1e-10: the oracle's iteration count and the FP64
    solution of the coloured-sweep solve."""
    dim, k, n = 2, 2, 64
    P = tps.PoissonProblem(dim, k, n)
    b = interior_random(dim, n * k + 1, 7)
    MG = tps.MultigridSolvers(P)
    x_ref, rep_ref = MG.solve_cg(torch.tensor(b, device="cuda"), precision="fp64", rel_tol=1e-12)
    P.set_smoother_kind("additive")
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    H.set_additive(0.25)
    xo, it_o, _ = H.solve_cg(b, precision=0, symmetric=True, rel_tol=1e-10)
    for precision in ("fp64", "fp32"):
        x, rep = MG.solve_cg(torch.tensor(b, device="cuda"), precision=precision, rel_tol=1e-10)
        assert rep.converged and rep.final_residual <= 1e-10
        assert abs(rep.iterations - it_o) <= 1, (precision, rep.iterations, it_o)
        assert relerr(x.cpu().numpy(), x_ref.cpu().numpy()) < 1e-8
    # back to the coloured sweep: the original solve
    P.set_smoother_kind("fused")
    x2, rep2 = MG.solve_cg(torch.tensor(b, device="cuda"), precision="fp64", rel_tol=1e-12)
    assert rep2.iterations == rep_ref.iterations
    with pytest.raises(tps.TpsError):
        P.set_smoother_kind("additive", 0.5)  # not below 2/2^dim
    P.close()
