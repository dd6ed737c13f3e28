"""GPU tests of the full-multigrid driver (tps_fmg, MultigridSolvers::solve of
include/solver.cuh:1784-1860) against the CPU oracle's restatement and on a
manufactured problem with inhomogeneous Dirichlet data."""
import math

import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import problems

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def level_rhs(dim, k, P, seed=0):
    return [problems.sine_modes_rhs(dim, k, P.cells(l), seed, 8, "cuda") for l in range(P.n_levels)]


@pytest.mark.parametrize("dim,k,n,n_coarse", [(3, 2, 16, 2), (2, 3, 32, 2), (3, 3, 12, 3)])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("fp32", 2e-5)])
@pytest.mark.parametrize("n_cycles", [1, 2])
def test_fmg_matches_oracle(cuda, oracle, dim, k, n, n_coarse, precision, tol, n_cycles):
    P = tps.PoissonProblem(dim, k, n, n_coarse=n_coarse)
    rhs = level_rhs(dim, k, P)
    x, rep = tps.MultigridSolvers(P).solve_fmg(rhs, precision=precision, n_cycles=n_cycles)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    ref = H.fmg([r.cpu().numpy() for r in rhs], precision=0 if precision == "fp64" else 1, n_cycles=n_cycles)
    assert relerr(x.cpu().numpy(), ref) < tol
    assert rep.iterations == n_cycles and 0 < rep.final_residual < 1e-1
    P.close()


def manufactured(P, dim, k, level):
    """u = prod sin(pi x_d) + (1 + x + 2y [+ 3z]) (harmonic affine part):
    f = dim pi^2 prod sin(pi x_d); nodal u_D on the boundary, zero inside."""
    n = P.cells(level)
    N1 = n * k + 1
    nodes = np.array([(c + t) / n for c in range(n) for t in problems.gauss_lobatto(k)[:-1]] + [1.0])
    grids = np.meshgrid(*([nodes] * dim), indexing="ij")[::-1]  # x fastest: arrays indexed [z][y][x]
    xs = [g for g in grids]  # xs[0] = x coordinate, xs[1] = y, ...
    u = np.ones_like(xs[0])
    for d in range(dim):
        u = u * np.sin(math.pi * xs[d])
    u = u + 1.0 + sum((d + 1) * xs[d] for d in range(dim))
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    bnd = np.any((idx == 0) | (idx == N1 - 1), axis=0)
    ud = np.where(bnd, u.reshape(-1), 0.0)
    l1 = problems.load_1d_sin(k, n, 1)
    load = l1
    for _ in range(dim - 1):
        load = np.kron(load, l1)
    f = dim * math.pi ** 2 * load
    return u.reshape(-1), ud, f


def boundary_mask(dim, N1):
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    return torch.tensor(np.any((idx == 0) | (idx == N1 - 1), axis=0), device="cuda")


@pytest.mark.parametrize("dim,k,n", [(3, 2, 16), (2, 4, 32)])
def test_fmg_inhomogeneous_dirichlet(cuda, oracle, dim, k, n):
    P = tps.PoissonProblem(dim, k, n)
    rhs, bnd = [], []
    for l in range(P.n_levels):
        _, ud, f = manufactured(P, dim, k, l)
        ud_t = torch.tensor(ud, device="cuda")
        aud = torch.empty_like(ud_t)
        tps.LaplaceOperator(P, level=l).vmult(aud, ud_t)  # interior rows: A u_D
        r = torch.tensor(f, device="cuda") - aud
        r[boundary_mask(dim, P.cells(l) * k + 1)] = 0.0
        rhs.append(r)  # constrained rows are zero, as the reference assembles them
        bnd.append(ud_t)
    MG = tps.MultigridSolvers(P)
    x2, rep2 = MG.solve_fmg(rhs, bnd, precision="fp64", n_cycles=2)
    # the exact discrete solution: homogeneous CG on the lifted right-hand side + u_D
    u0, _ = MG.solve_cg(rhs[-1], precision="fp64", rel_tol=1e-13)
    uh = (u0 + bnd[-1]).cpu().numpy()
    u_exact, _, _ = manufactured(P, dim, k, P.n_levels - 1)
    assert relerr(x2.cpu().numpy(), uh) < 1e-4
    # Dirichlet data are written into the boundary exactly
    idx = np.stack(np.unravel_index(np.arange(uh.size), (n * k + 1,) * dim))
    b = np.any((idx == 0) | (idx == n * k), axis=0)
    assert np.array_equal(x2.cpu().numpy()[b], bnd[-1].cpu().numpy()[b])
    # discretization accuracy: the FMG solution is as close to u as u_h is
    e_fmg = np.abs(x2.cpu().numpy() - u_exact).max()
    e_h = np.abs(uh - u_exact).max()
    assert e_fmg <= 1.5 * e_h + 1e-12
    # parity with the oracle's FMG on the same data
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels)
    ref = H.fmg([r.cpu().numpy() for r in rhs], [v.cpu().numpy() for v in bnd], precision=0, n_cycles=2)
    assert relerr(x2.cpu().numpy(), ref) < 1e-11
    P.close()
