"""Seeded synthetic right-hand sides for the benchmark configurations.

There is no public dataset for this path; the workloads are generated from a
seed with the shapes and value distributions the configurations name:

* ``nodal_uniform`` -- f = i.i.d. U[-1,1] nodal values, b = M_h f
  (2D Q2 64^2 configuration);
* ``sine_modes``    -- f = sum_j a_j sin(k_j pi x) sin(l_j pi y) sin(m_j pi z),
  a_j ~ U[-1,1], (k_j,l_j,m_j) ~ U{1..8}^3, b_i = int f phi_i with QGauss(k+1)
  (3D Q4 64^3 configuration; the quadrature follows
  LaplaceOperator::compute_residual, include/laplace_operator.cuh:118-181);
* ``nodal_normal``  -- f = i.i.d. N(0,1) nodal values, b = M_h f (3D Q7 32^3).

Dirichlet rows of b are zero.  The vectors are assembled with torch on the
device (input preparation only; not part of any timed solve).
"""
from __future__ import annotations

import numpy as np
import torch


def gauss_lobatto(k: int) -> np.ndarray:
    """k+1 Gauss-Lobatto points on [0,1] (FE_Q support points)."""
    if k == 1:
        return np.array([0.0, 1.0])
    inner = np.polynomial.legendre.Legendre.basis(k).deriv().roots()
    return np.concatenate([[0.0], np.sort(0.5 * (inner + 1.0)), [1.0]])


def lagrange_matrix(nodes: np.ndarray, x: np.ndarray) -> np.ndarray:
    """V[q, i] = phi_i(x_q) for the Lagrange basis on nodes."""
    V = np.ones((len(x), len(nodes)))
    for i, xi in enumerate(nodes):
        for m, xm in enumerate(nodes):
            if m != i:
                V[:, i] *= (x - xm) / (xi - xm)
    return V


def mass_1d(k: int, n: int) -> np.ndarray:
    """Global 1D mass matrix of n cells on [0,1] (dense, (nk+1)^2)."""
    nodes = gauss_lobatto(k)
    xq, wq = np.polynomial.legendre.leggauss(k + 1)
    xq = 0.5 * (xq + 1.0)
    wq = 0.5 * wq
    V = lagrange_matrix(nodes, xq)
    Mc = (V * wq[:, None]).T @ V / n
    N1 = n * k + 1
    M = np.zeros((N1, N1))
    for c in range(n):
        M[c * k:c * k + k + 1, c * k:c * k + k + 1] += Mc
    return M


def load_1d_sin(k: int, n: int, freq: int) -> np.ndarray:
    """b_i = int_0^1 sin(freq pi x) phi_i(x) dx with QGauss(k+1) per cell."""
    nodes = gauss_lobatto(k)
    xq, wq = np.polynomial.legendre.leggauss(k + 1)
    xq = 0.5 * (xq + 1.0)
    wq = 0.5 * wq
    V = lagrange_matrix(nodes, xq)
    N1 = n * k + 1
    b = np.zeros(N1)
    h = 1.0 / n
    for c in range(n):
        xs = (c + xq) * h
        b[c * k:c * k + k + 1] += V.T @ (wq * h * np.sin(freq * np.pi * xs))
    return b


def _zero_boundary(b: torch.Tensor, dim: int, N1: int) -> torch.Tensor:
    v = b.view((N1,) * dim)
    if dim == 2:
        v[0, :] = 0
        v[-1, :] = 0
        v[:, 0] = 0
        v[:, -1] = 0
    else:
        v[0] = 0
        v[-1] = 0
        v[:, 0] = 0
        v[:, -1] = 0
        v[:, :, 0] = 0
        v[:, :, -1] = 0
    return b


def apply_mass(f: torch.Tensor, dim: int, k: int, n: int) -> torch.Tensor:
    """b = (M1 (x) ... (x) M1) f with the global 1D mass matrix (lexicographic, x fastest)."""
    N1 = n * k + 1
    M = torch.tensor(mass_1d(k, n), dtype=f.dtype, device=f.device)
    v = f.view((N1,) * dim)
    if dim == 2:  # v[y, x]
        out = M @ v @ M.T
    else:  # v[z, y, x]
        out = torch.einsum("ab,zyb->zya", M, v)
        out = torch.einsum("ab,zbx->zax", M, out)
        out = torch.einsum("ab,byx->ayx", M, out)
    return out.reshape(-1).contiguous()


def nodal_rhs(dim: int, k: int, n: int, seed: int, dist: str = "uniform",
              device="cuda") -> torch.Tensor:
    rng = np.random.default_rng(seed)
    N1 = n * k + 1
    size = N1 ** dim
    f = rng.uniform(-1.0, 1.0, size) if dist == "uniform" else rng.standard_normal(size)
    ft = _zero_boundary(torch.tensor(f, dtype=torch.float64, device=device), dim, N1)
    return _zero_boundary(apply_mass(ft, dim, k, n), dim, N1)


def sine_modes_rhs(dim: int, k: int, n: int, seed: int, n_modes: int = 8,
                   device="cuda") -> torch.Tensor:
    rng = np.random.default_rng(seed)
    amps = rng.uniform(-1.0, 1.0, n_modes)
    freqs = rng.integers(1, 9, size=(n_modes, dim))
    N1 = n * k + 1
    b = torch.zeros((N1,) * dim, dtype=torch.float64, device=device)
    for a, fr in zip(amps, freqs):
        vs = [torch.tensor(load_1d_sin(k, n, int(f)), dtype=torch.float64, device=device) for f in fr]
        if dim == 2:  # b[y, x]
            b += a * torch.outer(vs[1], vs[0])
        else:  # b[z, y, x]
            b += a * torch.einsum("z,y,x->zyx", vs[2], vs[1], vs[0])
    return _zero_boundary(b.reshape(-1).contiguous(), dim, N1)


def interior_dofs(dim: int, k: int, n: int) -> int:
    return (n * k - 1) ** dim


WORKLOADS = {
    # name: (dim, k, n_cells, generator)
    "poisson2d_q2_64": (2, 2, 64, lambda d, k, n, s, dev: nodal_rhs(d, k, n, s, "uniform", dev)),
    "poisson3d_q4_64": (3, 4, 64, lambda d, k, n, s, dev: sine_modes_rhs(d, k, n, s, 8, dev)),
    "poisson3d_q7_32": (3, 7, 32, lambda d, k, n, s, dev: nodal_rhs(d, k, n, s, "normal", dev)),
}


def make_rhs(name: str, seed: int = 0, device="cuda", n_cells: int | None = None) -> torch.Tensor:
    dim, k, n, gen = WORKLOADS[name]
    return gen(dim, k, n if n_cells is None else n_cells, seed, device)
