"""Generates tests/golden/golden.npz: independent numpy/scipy computations of
every quantity the CPU oracle restates, used to pin the oracle.

The reference (LuciaZhang9/GPUTensorProductSmoother) ships no golden vectors
and cannot run here (deal.II with CUDA+MPI, CMakeLists.txt:81-102), so these
fixtures come from dense linear algebra on the definitions instead:

* 1D data: Gauss-Lobatto nodes (roots of P_k'), QGauss(k+1) cell mass and
  stiffness, patch matrices, interior generalized eigenvalues (scipy eigh),
  1D prolongation (coarse Lagrange basis at the child nodes);
* 2D/3D dense operators on small meshes: A = Kronecker sum of the global 1D
  matrices with identity Dirichlet rows (LaplaceOperator::vmult semantics,
  include/laplace_operator.cuh:86-101);
* one coloured patch sweep computed with dense local solves
  x_I <- A_II^{-1}(b_I - A_IB x_B) per patch, colours in the reference order
  (include/patch_base.template.cuh:1208-1285);
* prolongation/restriction as dense interpolation matrices (P and P^T with
  Dirichlet rows/columns removed, include/cuda_mg_transfer.template.cuh:561-706);
* a dense two-grid/three-grid V-cycle (include/solver.cuh:1952-2001).

Run:  python tests/golden/make_golden.py
"""
import os

import numpy as np
import scipy.linalg as sla

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def gl_nodes(k):
    if k == 1:
        return np.array([0.0, 1.0])
    r = np.polynomial.legendre.Legendre.basis(k).deriv().roots()
    return np.concatenate([[0.0], np.sort((r + 1) / 2), [1.0]])


def lagrange(nodes, x):
    V = np.ones((len(x), len(nodes)))
    D = np.zeros((len(x), len(nodes)))
    for i, xi in enumerate(nodes):
        others = [xm for m, xm in enumerate(nodes) if m != i]
        den = np.prod([xi - xm for xm in others])
        V[:, i] = np.prod([x - xm for xm in others], axis=0) / den
        d = np.zeros(len(x))
        for a in range(len(others)):
            d += np.prod([x - others[b] for b in range(len(others)) if b != a], axis=0)
        D[:, i] = d / den
    return V, D


def cell_matrices(k):
    xq, wq = np.polynomial.legendre.leggauss(k + 1)
    xq, wq = (xq + 1) / 2, wq / 2
    V, D = lagrange(gl_nodes(k), xq)
    return (V * wq[:, None]).T @ V, (D * wq[:, None]).T @ D


def prolongation_1d(k):
    nodes = gl_nodes(k)
    xf = np.concatenate([nodes / 2, 0.5 + nodes[1:] / 2])
    V, _ = lagrange(nodes, xf)
    V[np.abs(V) < 1e-14] = 0.0
    return V


def global_1d(k, n):
    Mc, Lc = cell_matrices(k)
    N1 = n * k + 1
    M = np.zeros((N1, N1))
    L = np.zeros((N1, N1))
    for c in range(n):
        s = slice(c * k, c * k + k + 1)
        M[s, s] += Mc / n
        L[s, s] += Lc * n
    return M, L


def global_operator(dim, k, n):
    M, L = global_1d(k, n)
    if dim == 2:
        A = np.kron(M, L) + np.kron(L, M)
    else:
        A = np.kron(np.kron(M, M), L) + np.kron(np.kron(M, L), M) + np.kron(np.kron(L, M), M)
    N1 = n * k + 1
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    bnd = np.any((idx == 0) | (idx == N1 - 1), axis=0)
    return A, bnd


def constrained(A, bnd):
    """identity Dirichlet rows, boundary columns kept (src is not zeroed)"""
    Ac = A.copy()
    Ac[bnd, :] = 0.0
    Ac[bnd, bnd] = 1.0
    return Ac


def patch_sweep(dim, k, n, x, b, A):
    N1 = n * k + 1
    npd = n - 1
    x = x.copy()
    for color in range(1 << dim):
        par = [(color >> d) & 1 for d in range(dim)]
        starts = [range(p, npd, 2) for p in par]
        grids = np.meshgrid(*starts, indexing="ij")
        pts = np.stack([g.ravel() for g in grids], axis=1) if grids[0].size else np.zeros((0, dim), int)
        new = {}
        for pp in pts:  # pp = (px, py[, pz])
            rng = [np.arange(pp[d] * k, pp[d] * k + 2 * k + 1) for d in range(dim)]
            box = np.meshgrid(*rng[::-1], indexing="ij")  # z, y, x order
            coords = np.stack([bx.ravel() for bx in box[::-1]], axis=1)  # x, y, z
            lin = sum(coords[:, d] * N1 ** d for d in range(dim))
            loc = coords - np.array([pp[d] * k for d in range(dim)])
            interior = np.all((loc > 0) & (loc < 2 * k), axis=1)
            I = lin[interior]
            B = lin[~interior]
            AII = A[np.ix_(I, I)]
            AIB = A[np.ix_(I, B)]
            new[tuple(pp)] = (I, np.linalg.solve(AII, b[I] - AIB @ x[B]))
        for I, v in new.values():
            x[I] = v
    return x


def prolongation_matrix(dim, k, nc):
    P1 = np.zeros((2 * nc * k + 1, nc * k + 1))
    p = prolongation_1d(k)
    for c in range(nc):
        P1[2 * c * k:2 * c * k + 2 * k + 1, c * k:c * k + k + 1] = p
    P = P1
    for _ in range(dim - 1):
        P = np.kron(P, P1)
    Nf, Nc = (2 * nc * k + 1) ** dim, (nc * k + 1) ** dim
    _, bf = global_operator(dim, k, 2 * nc)
    _, bc = global_operator(dim, k, nc)
    P = P.copy()
    P[bf, :] = 0.0
    P[:, bc] = 0.0
    return P


def main():
    out = {}
    for k in range(1, 8):
        Mc, Lc = cell_matrices(k)
        out[f"nodes_k{k}"] = gl_nodes(k)
        out[f"cmass_k{k}"] = Mc
        out[f"clap_k{k}"] = Lc
        out[f"prol_k{k}"] = prolongation_1d(k)
        n1 = 2 * k + 1
        Mp = np.zeros((n1, n1))
        Lp = np.zeros((n1, n1))
        for c in range(2):
            Mp[c * k:c * k + k + 1, c * k:c * k + k + 1] += Mc
            Lp[c * k:c * k + k + 1, c * k:c * k + k + 1] += Lc
        out[f"pmass_k{k}"] = Mp
        out[f"plap_k{k}"] = Lp
        h = 0.25
        lam = sla.eigh(Lp[1:-1, 1:-1] / h, Mp[1:-1, 1:-1] * h, eigvals_only=True)
        out[f"patch_eval_k{k}_h0.25"] = np.sort(lam)
    rng = np.random.default_rng(2024)
    for dim, k, n in [(2, 2, 4), (2, 3, 4), (3, 1, 4), (3, 2, 4)]:
        tag = f"d{dim}k{k}n{n}"
        A, bnd = global_operator(dim, k, n)
        N = A.shape[0]
        x = rng.uniform(-1, 1, N)
        b = rng.uniform(-1, 1, N)
        out[f"op_src_{tag}"] = x
        out[f"op_dst_{tag}"] = constrained(A, bnd) @ x
        out[f"sm_x_{tag}"] = x
        out[f"sm_b_{tag}"] = b
        out[f"sm_out_{tag}"] = patch_sweep(dim, k, n, x, b, A)
        nc = n // 2
        P = prolongation_matrix(dim, k, nc)
        c = rng.uniform(-1, 1, P.shape[1])
        f = rng.uniform(-1, 1, P.shape[0])
        out[f"tr_coarse_{tag}"] = c
        out[f"tr_fine_{tag}"] = f
        out[f"tr_prol_{tag}"] = f + P @ c
        out[f"tr_restr_{tag}"] = c + P.T @ f
        # dense two-level V-cycle: pre-sweep (zero start), restrict, exact coarse, prolongate, post-sweep
        Ac, bc_ = global_operator(dim, k, nc)
        d = rng.uniform(-1, 1, N)
        d[bnd] = 0.0
        su = patch_sweep(dim, k, n, np.zeros(N), d, A)
        t = d - constrained(A, bnd) @ su
        t[bnd] = 0.0
        dc = P.T @ t
        dc[bc_] = 0.0
        Ic = ~bc_
        sc = np.zeros(Ac.shape[0])
        sc[Ic] = np.linalg.solve(Ac[np.ix_(Ic, Ic)], dc[Ic])
        su = su + P @ sc
        su = patch_sweep(dim, k, n, su, d, A)
        out[f"vc_in_{tag}"] = d
        out[f"vc_out_{tag}"] = su
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, sum(v.size for v in out.values()), "values")


if __name__ == "__main__":
    main()
