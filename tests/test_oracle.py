"""CPU tests of the oracle: pinned against the independent golden fixtures
(tests/golden/make_golden.py) and against mathematical known answers.  No GPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("k", range(1, 8))
def test_1d_tables_match_golden(oracle, golden, k):
    nodes, m, l, p = oracle.fe1d(k)
    assert rel(nodes, golden[f"nodes_k{k}"]) < 1e-13
    assert rel(m, golden[f"cmass_k{k}"]) < 1e-13
    assert rel(l, golden[f"clap_k{k}"]) < 1e-13
    assert rel(p, golden[f"prol_k{k}"]) < 1e-13
    pm, pl = oracle.patch_matrices(k)
    assert rel(pm, golden[f"pmass_k{k}"]) < 1e-13
    assert rel(pl, golden[f"plap_k{k}"]) < 1e-13
    S, lam = oracle.patch_eigen(k, 0.25)
    assert rel(np.sort(lam), golden[f"patch_eval_k{k}_h0.25"]) < 1e-12


GCASES = [(2, 2, 4), (2, 3, 4), (3, 1, 4), (3, 2, 4)]


@pytest.mark.parametrize("dim,k,n", GCASES)
def test_level_ops_match_golden(oracle, golden, dim, k, n):
    t = f"d{dim}k{k}n{n}"
    assert rel(oracle.laplace_vmult(dim, k, n, golden["op_src_" + t]), golden["op_dst_" + t]) < 1e-13
    assert rel(oracle.smoother_step(dim, k, n, golden["sm_x_" + t], golden["sm_b_" + t]),
               golden["sm_out_" + t]) < 1e-12
    assert rel(oracle.prolongate_add(dim, k, n // 2, golden["tr_fine_" + t], golden["tr_coarse_" + t]),
               golden["tr_prol_" + t]) < 1e-13
    assert rel(oracle.restrict_add(dim, k, n // 2, golden["tr_coarse_" + t], golden["tr_fine_" + t]),
               golden["tr_restr_" + t]) < 1e-13
    H = oracle.Hierarchy(dim, k, 2, 2)
    assert rel(H.vcycle(golden["vc_in_" + t], precision=0), golden["vc_out_" + t]) < 1e-12


@pytest.mark.parametrize("k", range(1, 8))
def test_fd_eigenpairs_normalised(oracle, k):
    """V^T M V = I and V^T L V = diag(lambda) on the patch interior."""
    h = 1.0 / 8
    S, lam = oracle.patch_eigen(k, h)
    pm, pl = oracle.patch_matrices(k)
    MI, LI = h * pm[1:-1, 1:-1], pl[1:-1, 1:-1] / h
    assert np.allclose(S.T @ MI @ S, np.eye(2 * k - 1), atol=1e-10)
    assert np.allclose(S.T @ LI @ S, np.diag(lam), atol=1e-8 * lam.max())


@pytest.mark.parametrize("dim,k", [(2, 1), (2, 3), (3, 2), (3, 3)])
def test_restriction_is_transpose_of_prolongation(oracle, dim, k):
    nc = 2
    Nc, Nf = (nc * k + 1) ** dim, (2 * nc * k + 1) ** dim
    P = np.stack([oracle.prolongate_add(dim, k, nc, np.zeros(Nf), np.eye(Nc)[j]) for j in range(Nc)], 1)
    R = np.stack([oracle.restrict_add(dim, k, nc, np.zeros(Nc), np.eye(Nf)[j]) for j in range(Nf)], 1)
    assert np.abs(R - P.T).max() == 0.0


@pytest.mark.parametrize("dim,k", [(2, 2), (2, 4), (3, 3)])
def test_prolongation_reproduces_polynomials(oracle, dim, k):
    """Q_k interpolation is exact for polynomials of degree k vanishing on the boundary."""
    nc = 2
    def grid(n):
        x = np.linspace(0, 1, n * k + 1)  # node positions are not equispaced, but
        return x                            # the bubble below is sampled at true nodes
    nodes = np.concatenate([[0.0]] + [c / nc + oracle.fe1d(k)[0][1:] / nc for c in range(nc)])
    nodes_f = np.concatenate([[0.0]] + [c / (2 * nc) + oracle.fe1d(k)[0][1:] / (2 * nc)
                                        for c in range(2 * nc)])
    f1 = lambda x: x * (1 - x) * (0.3 + x) ** (k - 2) if k >= 2 else x * 0
    if k < 2:
        pytest.skip("needs k >= 2 for an interior-vanishing polynomial")
    def sample(nodes):
        g = [f1(nodes)] * dim
        v = g[0]
        for d in range(1, dim):
            v = np.multiply.outer(g[d], v)
        return v.ravel()
    c = sample(nodes)
    f = oracle.prolongate_add(dim, k, nc, np.zeros(len(nodes_f) ** dim), c)
    assert rel(f, sample(nodes_f)) < 1e-12


@pytest.mark.parametrize("dim,k", [(2, 2), (3, 2), (3, 3)])
def test_single_patch_smoother_is_exact_solve(oracle, dim, k):
    """On a 2-cell mesh the one vertex patch covers every interior DoF
    (the reference's coarse solver, include/solver.cuh:80-102)."""
    n = 2
    N1 = n * k + 1
    N = N1 ** dim
    A = np.stack([oracle.laplace_vmult(dim, k, n, np.eye(N)[j]) for j in range(N)], 1)
    idx = np.stack(np.unravel_index(np.arange(N), (N1,) * dim))
    I = ~np.any((idx == 0) | (idx == N1 - 1), axis=0)
    b = np.random.default_rng(1).uniform(-1, 1, N)
    b[~I] = 0
    x = oracle.smoother_step(dim, k, n, np.zeros(N), b, zero_init=True)
    assert rel(x[I], np.linalg.solve(A[np.ix_(I, I)], b[I])) < 1e-12
    assert np.all(np.linalg.eigvalsh(0.5 * (A[np.ix_(I, I)] + A[np.ix_(I, I)].T)) > 0)


def test_fp32_level_ops_close_to_fp64(oracle):
    dim, k, n = 3, 3, 4
    N = (n * k + 1) ** dim
    rng = np.random.default_rng(3)
    x, b = rng.uniform(-1, 1, N), rng.uniform(-1, 1, N)
    s64 = oracle.smoother_step(dim, k, n, x, b)
    s32 = oracle.smoother_step(dim, k, n, x.astype(np.float32), b.astype(np.float32))
    assert rel(s32, s64) < 1e-4


@pytest.mark.parametrize("k", [1, 2, 3])
def test_manufactured_solution_converges(oracle, k):
    """u = prod sin(3 pi x_d) (apps/poisson.cu:42-87): nodal error decays at
    O(h^(k+1)) or better in 2D."""
    errs = []
    for n in (8, 16):
        N1 = n * k + 1
        H = oracle.Hierarchy(2, k, 2, int(np.log2(n)))
        # load vector with a high-order quadrature per cell
        nodes = oracle.fe1d(k)[0]
        xq, wq = np.polynomial.legendre.leggauss(k + 4)
        xq, wq = (xq + 1) / 2, wq / 2
        V = np.ones((len(xq), k + 1))
        for i in range(k + 1):
            for m in range(k + 1):
                if m != i:
                    V[:, i] *= (xq - nodes[m]) / (nodes[i] - nodes[m])
        b1 = np.zeros(N1)
        for c in range(n):
            xs = (c + xq) / n
            b1[c * k:c * k + k + 1] += V.T @ (wq / n * np.sin(3 * np.pi * xs))
        b = 2 * (3 * np.pi) ** 2 * np.outer(b1, b1).ravel()
        idx = np.stack(np.unravel_index(np.arange(N1 ** 2), (N1,) * 2))
        b[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0
        x, it, _ = H.solve_cg(b, rel_tol=1e-12, max_it=200)
        xn = np.concatenate([[0.0]] + [c / n + nodes[1:] / n for c in range(n)])
        u = np.outer(np.sin(3 * np.pi * xn), np.sin(3 * np.pi * xn)).ravel()
        errs.append(np.abs(x - u).max())
    rate = np.log2(errs[0] / errs[1])
    assert rate > k + 0.5, (errs, rate)


@pytest.mark.parametrize("dim,k,nl", [(2, 2, 4), (3, 2, 3)])
def test_krylov_drivers_converge(oracle, dim, k, nl):
    H = oracle.Hierarchy(dim, k, 2, nl)
    N1 = (2 << (nl - 1)) * k + 1
    b = np.random.default_rng(5).uniform(-1, 1, N1 ** dim)
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    b[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0
    x, it, hist = H.solve_cg(b, precision=0, rel_tol=1e-10)
    assert np.linalg.norm(b - H.vmult(x)) <= 1.01e-10 * np.linalg.norm(b) and it < 15
    x32, it32, _ = H.solve_cg(b, precision=1, rel_tol=1e-10)
    assert it32 <= it + 1 and rel(x32, x) < 1e-8
    xg, itg, _ = H.solve_gmres(b, precision=2, reduce=1e-9)
    assert itg <= 20 and rel(xg, x) < 1e-6


def test_dense_coarse_solve_for_three_cell_mesh(oracle):
    H = oracle.Hierarchy(3, 2, 3, 2)  # 3 and 6 cells per direction
    Nc = oracle.ndofs(3, 2, 3)
    N1 = 3 * 2 + 1
    b = np.random.default_rng(7).uniform(-1, 1, Nc)
    idx = np.stack(np.unravel_index(np.arange(Nc), (N1,) * 3))
    b[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0
    x = H.coarse_solve(b)
    assert rel(oracle.laplace_vmult(3, 2, 3, x), b) < 1e-11


def test_oracle_adjoint_matches_finite_differences(oracle):
    """The FP64 oracle adjoint (the reference the GPU adjoint is checked
    against) agrees with central differences of its own solves (h = 1e-6)."""
    dim, k, nc, nl = 3, 2, 2, 2
    n = nc * 2 ** (nl - 1)
    N1 = n * k + 1
    rng = np.random.default_rng(21)
    kap = np.exp(rng.normal(0.0, 0.5, n ** dim))
    f = rng.standard_normal(N1 ** dim)

    def solve(f_, k_):
        H = oracle.Hierarchy(dim, k, nc, nl, kappa=k_)
        b = oracle.zero_dirichlet(oracle.mass_vmult(dim, k, n, f_), dim, N1)
        return H.solve_cg(b, precision=0, rel_tol=1e-14, max_it=400)[0]

    u0 = solve(f, kap)
    ut = u0 * (1.0 + 0.3 * rng.standard_normal(N1 ** dim))

    def J(f_, k_):
        return 0.5 * np.sum((solve(f_, k_) - ut) ** 2)

    _, gf, gk = oracle.adjoint_gradients(dim, k, nc, nl, kap, f, ut, rel_tol=1e-14)
    h = 1e-6
    for _ in range(3):
        df = rng.standard_normal(N1 ** dim)
        dk = rng.standard_normal(n ** dim) * kap
        fd_f = (J(f + h * df, kap) - J(f - h * df, kap)) / (2 * h)
        fd_k = (J(f, kap + h * dk) - J(f, kap - h * dk)) / (2 * h)
        assert abs(gf @ df - fd_f) <= 1e-6 * abs(fd_f)
        assert abs(gk @ dk - fd_k) <= 1e-6 * abs(fd_k)


@pytest.mark.parametrize("dim,k,n", [(2, 2, 4), (3, 2, 4), (3, 3, 2)])
def test_oracle_cell_energy_and_mass(oracle, dim, k, n):
    """Per-cell energies sum to lam^T A u and equal the kappa-indicator
    operator of the oracle; the mass apply equals the dense Kronecker product
    of the global 1D mass matrices."""
    N1 = n * k + 1
    rng = np.random.default_rng(3)
    u = oracle.zero_dirichlet(rng.uniform(-1, 1, N1 ** dim), dim, N1)
    lam = oracle.zero_dirichlet(rng.uniform(-1, 1, N1 ** dim), dim, N1)
    e = oracle.cell_energy(dim, k, n, u, lam)
    tot = lam @ oracle.laplace_vmult(dim, k, n, u)
    assert abs(e.sum() - tot) <= 1e-13 * abs(tot)
    for c in (0, n ** dim - 1):
        ind = np.zeros(n ** dim)
        ind[c] = 1.0
        assert abs(e[c] - lam @ oracle.laplace_vmult(dim, k, n, u, kappa=ind)) <= 1e-13
    _, mass, _, _ = oracle.fe1d(k)
    M1 = np.zeros((N1, N1))
    for c in range(n):
        M1[c * k:c * k + k + 1, c * k:c * k + k + 1] += mass / n
    M = M1
    for _ in range(dim - 1):
        M = np.kron(M, M1)
    f = rng.uniform(-1, 1, N1 ** dim)
    assert np.abs(M @ f - oracle.mass_vmult(dim, k, n, f)).max() <= 1e-15


def _quad_points_np(dim, k, n):
    xq = 0.5 * (np.polynomial.legendre.leggauss(k + 1)[0] + 1.0)
    t = (np.arange(n)[:, None] + xq[None, :]) / n
    if dim == 2:
        xs = np.broadcast_to(t[None, :, None, :], (n, n, k + 1, k + 1))
        ys = np.broadcast_to(t[:, None, :, None], (n, n, k + 1, k + 1))
        return xs.reshape(n * n, -1), ys.reshape(n * n, -1)
    sh = (n, n, n, k + 1, k + 1, k + 1)
    xs = np.broadcast_to(t[None, None, :, None, None, :], sh)
    ys = np.broadcast_to(t[None, :, None, None, :, None], sh)
    zs = np.broadcast_to(t[:, None, None, :, None, None], sh)
    return xs.reshape(n ** 3, -1), ys.reshape(n ** 3, -1), zs.reshape(n ** 3, -1)


@pytest.mark.parametrize("dim,k,n", [(2, 2, 3), (2, 5, 2), (3, 2, 2), (3, 4, 2)])
def test_oracle_assemble_rhs_pinned(oracle, dim, k, n):
    """The assembly restatement is pinned twice: for f in Q_k (given at the
    Gauss points by interpolating nodal values) QGauss(k+1) is exact and
    b = M f; for the sine-mode right-hand side it equals the 1D-factorised
    assembly the benchmark inputs use."""
    import torch
    from gputensorproductsmoother_b200 import problems
    N1 = n * k + 1
    rng = np.random.default_rng(dim * 100 + k)
    fn = rng.uniform(-1, 1, N1 ** dim)
    V, _ = oracle._shape_at_gauss(k)
    F = fn.reshape((N1,) * dim)
    blocks = []
    for c in np.ndindex(*((n,) * dim)):
        sl = tuple(slice(ci * k, ci * k + k + 1) for ci in c)
        blk = F[sl]
        if dim == 2:
            blocks.append(np.einsum("qj,pi,ji->qp", V, V, blk).reshape(-1))
        else:
            blocks.append(np.einsum("rl,qj,pi,lji->rqp", V, V, V, blk).reshape(-1))
    b = oracle.assemble_rhs(dim, k, n, np.stack(blocks))
    ref = oracle.zero_dirichlet(oracle.mass_vmult(dim, k, n, fn), dim, N1)
    assert np.abs(b - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max())
    # sine modes: f = sum_j a_j prod_d sin(f_jd pi x_d), same seed as sine_modes_rhs
    rs = np.random.default_rng(5)
    amps = rs.uniform(-1.0, 1.0, 4)
    freqs = rs.integers(1, 9, size=(4, dim))
    pts = _quad_points_np(dim, k, n)
    fq = sum(a * np.prod([np.sin(int(fr[d]) * np.pi * pts[d]) for d in range(dim)], axis=0)
             for a, fr in zip(amps, freqs))
    bs = oracle.assemble_rhs(dim, k, n, fq)
    ref = problems.sine_modes_rhs(dim, k, n, 5, 4, device="cpu").numpy()
    assert np.abs(bs - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max())
