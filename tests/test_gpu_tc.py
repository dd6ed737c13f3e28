"""GPU tests of the tensor-core (tcgen05, TF32 operands, FP32 accumulation)
patch smoother: one sweep against the FP64 oracle sweep (TF32 tolerance), the
TF32 V-cycle inside the FP64 outer CG against the FP64 solve, and the
timing hook."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps

pytestmark = pytest.mark.gpu

# TF32 keeps 10 mantissa bits: one sweep deviates from the FP64 sweep by
# about 1e-3 of its largest entry (operands rounded to nearest between the
# eight contraction stages)
TF32_SWEEP_TOL = 1e-2


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def interior_random(N1, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, N1 ** 3)
    idx = np.stack(np.unravel_index(np.arange(N1 ** 3), (N1,) * 3))
    v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return v


@pytest.mark.parametrize("k,n", [(2, 8), (3, 4), (4, 4), (4, 8), (5, 4), (6, 4), (7, 4)])
@pytest.mark.parametrize("zero_init", [False, True])
def test_tc_sweep_matches_oracle(cuda, oracle, k, n, zero_init):
    P = tps.PoissonProblem(3, k, n)
    N1 = n * k + 1
    x0, b = interior_random(N1, 1), interior_random(N1, 2)
    ref = oracle.smoother_step(3, k, n, x0, b, zero_init=zero_init)
    x = torch.tensor(x0, dtype=torch.float32, device="cuda")
    S = tps.PatchSmoother(P, tensor_cores=True)
    (S.vmult if zero_init else S.step)(x, torch.tensor(b, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    got = x.cpu().numpy()
    assert np.all(np.isfinite(got))
    e = relerr(got, ref)
    assert e < TF32_SWEEP_TOL, e
    # the tensor-core sweep is a TF32 rounding of the same sweep, not another method
    assert e > 0.0
    mean = np.abs(got - ref).mean() / np.abs(ref).max()
    assert mean < TF32_SWEEP_TOL / 10, mean


@pytest.mark.parametrize("k,n", [(4, 8), (3, 16), (7, 4)])
def test_tc_vcycle_cg_reaches_fp64_solution(cuda, k, n):
    P = tps.PoissonProblem(3, k, n)
    b = torch.tensor(interior_random(n * k + 1, 3), device="cuda")
    MG = tps.MultigridSolvers(P)
    x64, r64 = MG.solve_cg(b, precision="fp64", rel_tol=1e-10)
    x32, r32 = MG.solve_cg(b, precision="fp32", rel_tol=1e-10)
    xtc, rtc = MG.solve_cg(b, precision="tf32", rel_tol=1e-10)
    assert rtc.converged and rtc.final_residual <= 1e-10
    assert relerr(xtc.cpu().numpy(), x64.cpu().numpy()) < 1e-8
    # the TF32 V-cycle is a slightly weaker preconditioner than the FP32 one
    assert rtc.iterations <= r32.iterations + 2, (rtc.iterations, r32.iterations, r64.iterations)


def test_tc_timing_hook(cuda):
    P = tps.PoissonProblem(3, 4, 16)
    ms = P.time_smoother(dtype="tf32", sweeps=3)
    assert ms > 0.0


# three-term TF32 split (a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32 accumulation):
# products to about FP32 accuracy, so a sweep meets the FP32 sweep tolerance
TF32X3_SWEEP_TOL = 2e-5


@pytest.mark.parametrize("n", [4, 8, 16])
@pytest.mark.parametrize("zero_init", [False, True])
def test_tf32x3_sweep_matches_oracle_at_fp32_accuracy(cuda, oracle, n, zero_init):
    """Degree 4 (the vector-producer patch-GEMM kernel): the three-pass
    tensor-core sweep agrees with the FP64 oracle sweep and with the FP32 SIMT
    sweep to the FP32 tolerance; the one-pass TF32 sweep of the same kernel
    stays within the TF32 tolerance."""
    k = 4
    P = tps.PoissonProblem(3, k, n)
    N1 = n * k + 1
    x0, b = interior_random(N1, 11), interior_random(N1, 12)
    ref = oracle.smoother_step(3, k, n, x0, b, zero_init=zero_init)
    bd = torch.tensor(b, dtype=torch.float32, device="cuda")
    out = {}
    for mode in ("tf32x3", "tf32", False):
        x = torch.tensor(x0, dtype=torch.float32, device="cuda")
        S = tps.PatchSmoother(P, tensor_cores=mode)
        (S.vmult if zero_init else S.step)(x, bd)
        torch.cuda.synchronize()
        out[mode] = x.cpu().numpy()
    assert np.all(np.isfinite(out["tf32x3"]))
    assert relerr(out["tf32x3"], ref) < TF32X3_SWEEP_TOL, relerr(out["tf32x3"], ref)
    assert relerr(out["tf32x3"], out[False]) < TF32X3_SWEEP_TOL
    assert relerr(out["tf32"], ref) < TF32_SWEEP_TOL


def test_tf32x3_vcycle_cg_matches_fp32_iterations(cuda):
    """The three-pass tensor-core V-cycle (degree 4) preconditions the FP64 CG
    like the FP32 V-cycle: same iteration count, solution within 1e-8 of the
    FP64-V-cycle solve."""
    P = tps.PoissonProblem(3, 4, 32)
    b = torch.tensor(interior_random(4 * 32 + 1, 13), device="cuda")
    MG = tps.MultigridSolvers(P)
    x64, r64 = MG.solve_cg(b, precision="fp64", rel_tol=1e-10)
    x32, r32 = MG.solve_cg(b, precision="fp32", rel_tol=1e-10)
    x3, r3 = MG.solve_cg(b, precision="tf32x3", rel_tol=1e-10)
    assert r3.converged and r3.final_residual <= 1e-10
    assert r3.iterations == r32.iterations
    assert relerr(x3.cpu().numpy(), x64.cpu().numpy()) < 1e-8


def test_tf32x3_other_degrees_unsupported(cuda):
    P = tps.PoissonProblem(3, 3, 8)
    x = P.new_vector(dtype=torch.float32)
    with pytest.raises(tps.TpsError):
        tps.PatchSmoother(P, tensor_cores="tf32x3").step(x, P.new_vector(dtype=torch.float32))
    # the V-cycle precision falls back to the FP32 smoother at other degrees
    b = torch.tensor(interior_random(3 * 8 + 1, 14), device="cuda")
    x3, r3 = tps.MultigridSolvers(P).solve_cg(b, precision="tf32x3", rel_tol=1e-10)
    assert r3.converged
