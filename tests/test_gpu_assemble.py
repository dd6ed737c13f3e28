"""Right-hand-side assembly on the device (tps_assemble_rhs) against the
oracle's numpy restatement of the QGauss(k+1) load-vector loop of
LaplaceOperator::compute_residual (include/laplace_operator.cuh:118-181).

FP64 throughout: random f at the Gauss points to 1e-13 relative (max norm),
the sine-mode right-hand side of the benchmark configurations to 1e-13, and
run-to-run bit identity (colour-by-colour accumulation, no atomics)."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import problems

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _rel_max(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("dim,k,n", [(2, 1, 5), (2, 2, 6), (2, 5, 4), (2, 7, 3),
                                     (3, 1, 4), (3, 2, 4), (3, 3, 3), (3, 4, 4), (3, 7, 2)])
def test_assemble_random_f_matches_oracle(cuda, oracle, dim, k, n):
    P = tps.PoissonProblem(dim, k, n)
    rng = np.random.default_rng(dim * 10 + k)
    fq = rng.uniform(-1, 1, (n ** dim, (k + 1) ** dim))
    b = P.assemble_rhs(torch.tensor(fq, device="cuda")).cpu().numpy()
    ref = oracle.assemble_rhs(dim, k, n, fq)
    assert _rel_max(b, ref) <= TOL, _rel_max(b, ref)
    # Dirichlet rows are zero, not just small
    N1 = n * k + 1
    v = b.reshape((N1,) * dim)
    for ax in range(dim):
        assert not np.take(v, [0, N1 - 1], axis=ax).any()
    P.close()


@pytest.mark.parametrize("dim,k,n", [(2, 2, 16), (3, 4, 8), (3, 3, 6)])
def test_assemble_sine_modes_matches_benchmark_rhs(cuda, dim, k, n):
    """f = sum_j a_j prod_d sin(f_jd pi x_d) evaluated at the device's own
    quadrature points reproduces the sine-mode right-hand side of the
    benchmark inputs (assembled there from 1D factors)."""
    P = tps.PoissonProblem(dim, k, n)
    rs = np.random.default_rng(7)
    amps = rs.uniform(-1.0, 1.0, 8)
    freqs = rs.integers(1, 9, size=(8, dim))

    def f(*xs):
        out = torch.zeros_like(xs[0])
        for a, fr in zip(amps, freqs):
            term = torch.full_like(xs[0], float(a))
            for d in range(dim):
                term = term * torch.sin(int(fr[d]) * np.pi * xs[d])
            out += term
        return out

    b = P.assemble_rhs(f).cpu().numpy()
    ref = problems.sine_modes_rhs(dim, k, n, 7, 8, device="cpu").numpy()
    assert _rel_max(b, ref) <= TOL, _rel_max(b, ref)
    P.close()


def test_assemble_deterministic_and_levels(cuda, oracle):
    P = tps.PoissonProblem(3, 4, 16)
    rng = np.random.default_rng(3)
    fq = torch.tensor(rng.uniform(-1, 1, (16 ** 3, 125)), device="cuda")
    b1 = P.assemble_rhs(fq)
    b2 = P.assemble_rhs(fq)
    assert torch.equal(b1, b2)
    # a coarser level of the same hierarchy
    lv = P.n_levels - 2
    nc = P.cells(lv)
    fc = rng.uniform(-1, 1, (nc ** 3, 125))
    bc = P.assemble_rhs(torch.tensor(fc, device="cuda"), level=lv).cpu().numpy()
    assert _rel_max(bc, oracle.assemble_rhs(3, 4, nc, fc)) <= TOL
    with pytest.raises(ValueError):
        P.assemble_rhs(fq[:-1])
    P.close()


def test_assembled_rhs_solves_to_manufactured_solution(cuda):
    """-Lap u = f with u = sin(pi x) sin(pi y) sin(pi z): assembling f on the
    device and solving with the FP64 V-cycle gives the Q4 discretisation error
    (nodal max error 1.8e-10 on 16^3 cells with the oracle; bound 1e-8)."""
    k, n = 4, 16
    P = tps.PoissonProblem(3, k, n)
    b = P.assemble_rhs(lambda x, y, z: 3 * np.pi ** 2 * torch.sin(np.pi * x) * torch.sin(np.pi * y)
                       * torch.sin(np.pi * z))
    x, rep = tps.MultigridSolvers(P).solve_cg(b, precision="fp64", rel_tol=1e-12)
    assert rep.converged
    nodes = problems.gauss_lobatto(k)
    g = np.concatenate([(c + nodes[:-1]) / n for c in range(n)] + [[1.0]])
    u = np.einsum("z,y,x->zyx", np.sin(np.pi * g), np.sin(np.pi * g), np.sin(np.pi * g)).reshape(-1)
    err = np.abs(x.cpu().numpy() - u).max()
    assert err < 1e-8, err
    P.close()
