"""GPU parity of every kernel of the hot path against the CPU oracle, through
the C ABI (libtps.so), on seeded inputs small enough for the oracle.

Tolerances: FP64 paths 1e-12 relative (max-norm), FP32 paths 2e-5 relative.
"""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def relerr(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def dev(a, dtype):
    return torch.tensor(np.asarray(a), dtype=dtype, device="cuda")


CASES = [(2, k, 4) for k in range(1, 8)] + [(2, 2, 8), (2, 3, 16)] + \
        [(3, k, 4) for k in range(1, 8)] + [(3, 2, 8), (3, 4, 8)]


@pytest.mark.parametrize("dim,k,n", CASES)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_laplace_vmult(cuda, oracle, dim, k, n, dtype):
    P = tps.PoissonProblem(dim, k, n)
    N = P.n_dofs()
    rng = np.random.default_rng(100 + 10 * dim + k)
    src = rng.uniform(-1, 1, N)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    ref = oracle.laplace_vmult(dim, k, n, src.astype(npdt))
    dst = P.new_vector(dtype=dtype)
    tps.LaplaceOperator(P).vmult(dst, dev(src, dtype))
    torch.cuda.synchronize()
    err = relerr(dst.cpu().numpy(), ref)
    assert err < (TOL64 if dtype == torch.float64 else TOL32), err


@pytest.mark.parametrize("dim,k,n", CASES)
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("zero_init,reverse", [(False, False), (True, False), (False, True)])
def test_smoother_step(cuda, oracle, dim, k, n, dtype, zero_init, reverse):
    P = tps.PoissonProblem(dim, k, n)
    N = P.n_dofs()
    rng = np.random.default_rng(200 + 10 * dim + k)
    x0 = rng.uniform(-1, 1, N)
    b = rng.uniform(-1, 1, N)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    ref = oracle.smoother_step(dim, k, n, x0.astype(npdt), b.astype(npdt), zero_init=zero_init,
                               reverse=reverse)
    x = dev(x0, dtype)
    sm = tps.PatchSmoother(P)
    if zero_init:
        sm.vmult(x, dev(b, dtype), reverse=reverse)
    else:
        sm.step(x, dev(b, dtype), reverse=reverse)
    torch.cuda.synchronize()
    err = relerr(x.cpu().numpy(), ref)
    assert err < (TOL64 if dtype == torch.float64 else TOL32), err


@pytest.mark.parametrize("dim,k,n", CASES)
@pytest.mark.parametrize("variant", ["separate", "global", "exact"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("zero_init,reverse", [(False, False), (True, True)])
def test_smoother_variants(cuda, oracle, dim, k, n, variant, dtype, zero_init, reverse):
    """The reference's SEPERATE, GLOBAL and Exact smoother variants (separate
    residual and local-solve kernels, written independently of the fused
    ones) give the oracle's sweep.  Exact in FP32 sums up to (2k-1)^3 products
    per entry of its dense inverse, hence the looser 1e-4."""
    if variant == "exact" and dim == 3 and k == 7 and (zero_init or dtype == torch.float32):
        pytest.skip("one 3D Q7 Exact case: its dense inverse takes ~5 s of host time per handle")
    P = tps.PoissonProblem(dim, k, n)
    N = P.n_dofs()
    rng = np.random.default_rng(300 + 10 * dim + k)
    x0 = rng.uniform(-1, 1, N)
    b = rng.uniform(-1, 1, N)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    ref = oracle.smoother_step(dim, k, n, x0.astype(npdt), b.astype(npdt), zero_init=zero_init,
                               reverse=reverse)
    x = dev(x0, dtype)
    sm = tps.PatchSmoother(P, variant=variant)
    (sm.vmult if zero_init else sm.step)(x, dev(b, dtype), reverse=reverse)
    torch.cuda.synchronize()
    err = relerr(x.cpu().numpy(), ref)
    tol = TOL64 if dtype == torch.float64 else (1e-4 if variant == "exact" else TOL32)
    assert err < tol, err
    # a second sweep continues from the first, as the fused one does
    ref2 = oracle.smoother_step(dim, k, n, ref.astype(npdt), b.astype(npdt), reverse=reverse)
    sm.step(x, dev(b, dtype), reverse=reverse)
    torch.cuda.synchronize()
    assert relerr(x.cpu().numpy(), ref2) < 4 * tol
    P.close()


def test_smoother_variant_errors(cuda):
    P = tps.PoissonProblem(3, 2, 4, kappa=np.ones(64))
    x = P.new_vector()
    with pytest.raises(tps.TpsError):
        tps.PatchSmoother(P, variant="global").step(x, P.new_vector())
    with pytest.raises(ValueError):
        tps.PatchSmoother(P, variant="nonsense")
    P.close()


@pytest.mark.parametrize("dim,k", [(2, k) for k in range(1, 8)] + [(3, k) for k in range(1, 8)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_transfer(cuda, oracle, dim, k, dtype):
    P = tps.PoissonProblem(dim, k, 8 if dim == 3 and k > 4 else 8)
    T = tps.MGTransferCUDA(P)
    lf = P.n_levels - 1
    nc = P.cells(lf - 1)
    rng = np.random.default_rng(300 + 10 * dim + k)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    coarse = rng.uniform(-1, 1, P.n_dofs(lf - 1))
    fine0 = rng.uniform(-1, 1, P.n_dofs(lf))
    ref = oracle.prolongate_add(dim, k, nc, fine0.astype(npdt), coarse.astype(npdt))
    fine = dev(fine0, dtype)
    T.prolongate_and_add(lf, fine, dev(coarse, dtype))
    torch.cuda.synchronize()
    tol = TOL64 if dtype == torch.float64 else TOL32
    assert relerr(fine.cpu().numpy(), ref) < tol
    coarse0 = rng.uniform(-1, 1, P.n_dofs(lf - 1))
    ref = oracle.restrict_add(dim, k, nc, coarse0.astype(npdt), fine0.astype(npdt))
    c = dev(coarse0, dtype)
    T.restrict_and_add(lf, c, dev(fine0, dtype))
    torch.cuda.synchronize()
    assert relerr(c.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("dim,k,n", [(2, 2, 16), (2, 4, 8), (3, 1, 8), (3, 2, 8), (3, 3, 8), (3, 4, 4)])
@pytest.mark.parametrize("precision,oprec,tol", [("fp64", 0, TOL64), ("fp32", 1, 1e-4),
                                                ("fp64_rounded", 2, TOL64)])
@pytest.mark.parametrize("symmetric", [False, True])
def test_vcycle(cuda, oracle, dim, k, n, precision, oprec, tol, symmetric):
    P = tps.PoissonProblem(dim, k, n)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    N = P.n_dofs()
    rng = np.random.default_rng(400 + 10 * dim + k)
    src = rng.uniform(-1, 1, N)
    ref = H.vcycle(src, precision=oprec, symmetric=symmetric)
    dst = P.new_vector()
    tps.MultigridSolvers(P).vmult(dst, dev(src, torch.float64), precision=precision,
                                  symmetric=symmetric)
    torch.cuda.synchronize()
    assert relerr(dst.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("k,n", [(2, 8), (3, 8), (4, 8), (5, 4), (6, 4), (7, 4)])
@pytest.mark.parametrize("precision,oprec,tol", [("fp64", 0, TOL64), ("fp32", 1, 1e-4)])
def test_vcycle_smoother_variants(cuda, oracle, k, n, precision, oprec, tol):
    """Every compiled 3D smoother variant (patches per CTA batch P, P/2, P/4,
    one warp per patch, two patches per warp in packed FP32) gives the
    oracle's V-cycle; the variants only regroup
    the independent patches of a colour with the same per-patch arithmetic,
    so their V-cycles are bit-identical."""
    P = tps.PoissonProblem(3, k, n)
    H = oracle.Hierarchy(3, k, P.n_coarse, P.n_levels)
    rng = np.random.default_rng(450 + k)
    src = rng.uniform(-1, 1, P.n_dofs())
    ref = H.vcycle(src, precision=oprec, symmetric=True)
    dt = "fp64" if precision == "fp64" else "fp32"
    variants = P.smoother_variants(dt)
    assert len(variants) == 5
    outs = []
    for v in range(len(variants)):
        P.set_smoother_variant(v, dt)
        assert P.smoother_variant(0, dt) == v
        dst = P.new_vector()
        tps.MultigridSolvers(P).vmult(dst, dev(src, torch.float64), precision=precision, symmetric=True)
        torch.cuda.synchronize()
        assert relerr(dst.cpu().numpy(), ref) < tol, (v, variants[v])
        outs.append(dst.cpu().numpy())
    for v in range(1, len(outs)):
        assert np.array_equal(outs[v], outs[0]), (v, variants[v], relerr(outs[v], outs[0]))
    P.close()


def _rhs(dim, N1, seed):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1, 1, N1 ** dim)
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    b[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return b


@pytest.mark.parametrize("dim,k,n", [(2, 2, 32), (3, 2, 8), (3, 4, 8), (3, 4, 6), (3, 4, 12), (3, 3, 6), (3, 7, 8)])
def test_cg_fp64_matches_oracle(cuda, oracle, dim, k, n):
    """FP64 CG through the C ABI against the oracle: identical iteration
    counts and residual histories.  The 3D cases include meshes of 3 * 2^L
    cells (dense coarse solve), whose finest level does not fill the
    operator's xy tiles (the fused q = A p and its partial p.q sums)."""
    P = tps.PoissonProblem(dim, k, n)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    b = _rhs(dim, n * k + 1, 7)
    xr, it_r, hist_r = H.solve_cg(b, precision=0, symmetric=True, rel_tol=1e-10)
    x, rep = tps.MultigridSolvers(P).solve_cg(dev(b, torch.float64), precision="fp64",
                                              symmetric=True, rel_tol=1e-10)
    assert rep.converged and rep.iterations == it_r
    xg = x.cpu().numpy()
    # the reference-parity bar: solution within 1e-12 relative (2-norm)
    assert np.linalg.norm(xg - xr) <= 1e-12 * np.linalg.norm(xr)
    assert relerr(xg, xr) < 1e-11
    np.testing.assert_allclose(rep.history, hist_r, rtol=1e-6)


@pytest.mark.parametrize("dim,k,n", [(2, 2, 32), (3, 3, 8), (3, 4, 8)])
@pytest.mark.parametrize("use_graph", [True, False])
def test_cg_mixed_error_vs_fp64_oracle(cuda, oracle, dim, k, n, use_graph):
    P = tps.PoissonProblem(dim, k, n)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    b = _rhs(dim, n * k + 1, 8)
    xr, it_r, _ = H.solve_cg(b, precision=0, symmetric=True, rel_tol=1e-12, max_it=200)
    with torch.cuda.stream(torch.cuda.Stream()):
        x, rep = tps.MultigridSolvers(P).solve_cg(dev(b, torch.float64), precision="fp32",
                                                  rel_tol=1e-10, use_graph=use_graph)
        torch.cuda.synchronize()
    assert rep.converged
    # true residual of the GPU solution, computed by the oracle
    r = b - H.vmult(x.cpu().numpy())
    assert np.linalg.norm(r) <= 1.01e-10 * np.linalg.norm(b)
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr)


@pytest.mark.parametrize("dim,k,n", [(2, 2, 16), (3, 3, 8)])
def test_gmres_parity(cuda, oracle, dim, k, n):
    """deal.II-SolverGMRES semantics with the reference's FP32-rounded FP64
    V-cycle: identical iteration count and solution."""
    P = tps.PoissonProblem(dim, k, n)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    b = _rhs(dim, n * k + 1, 9)
    xr, it_r, hist_r = H.solve_gmres(b, precision=2, reduce=1e-9, abs_tol=1e-16, max_it=20)
    x, rep = tps.MultigridSolvers(P).solve_gmres(dev(b, torch.float64), precision="fp64_rounded",
                                                 max_iter=20, reduce=1e-9)
    assert rep.iterations == it_r
    assert relerr(x.cpu().numpy(), xr) < 1e-10


@pytest.mark.parametrize("k,n", [(4, 32), (3, 16), (5, 8)])
def test_pair_kernel_solve_bit_identical(cuda, k, n):
    """The two-patches-per-warp packed-FP32 smoother (variant 4) and the
    one-warp-per-patch kernel (variant 3, or the CTA batch where that is not
    compiled) give bit-identical FP32-V-cycle CG solves: same residual
    histories, same solution."""
    P = tps.PoissonProblem(3, k, n)
    b = dev(_rhs(3, n * k + 1, 31), torch.float64)
    MG = tps.MultigridSolvers(P)
    out = {}
    for v in (3, 4):
        P.set_smoother_variant(v, "fp32")
        x, rep = MG.solve_cg(b, precision="fp32", rel_tol=1e-10)
        torch.cuda.synchronize()
        out[v] = (x.clone(), list(rep.history), rep.iterations)
    assert out[3][2] == out[4][2]
    assert out[3][1] == out[4][1]
    assert torch.equal(out[3][0], out[4][0])
    P.close()
