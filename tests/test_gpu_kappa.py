"""GPU tests of the variable-coefficient path and the adjoint gradients
(no reference counterpart; checked against the CPU oracle, dense algebra and
central finite differences)."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def kappa_field(dim, n, seed):
    return np.exp(np.random.default_rng(seed).normal(0.0, 0.5, n ** dim))


def bvec(dim, N1, seed):
    b = np.random.default_rng(seed).uniform(-1, 1, N1 ** dim)
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    b[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return b


@pytest.mark.parametrize("dim,k,n", [(2, 2, 8), (2, 3, 4), (3, 2, 4), (3, 4, 4), (3, 3, 6)])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 2e-5)])
def test_kappa_level_ops(cuda, oracle, dim, k, n, dtype, tol):
    kap = kappa_field(dim, n, 1)
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    N = P.n_dofs()
    rng = np.random.default_rng(2)
    x0, b = rng.uniform(-1, 1, N), rng.uniform(-1, 1, N)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    ref = oracle.laplace_vmult(dim, k, n, x0.astype(npdt), kappa=kap)
    y = P.new_vector(dtype=dtype)
    tps.LaplaceOperator(P).vmult(y, torch.tensor(x0, dtype=dtype, device="cuda"))
    torch.cuda.synchronize()
    assert relerr(y.cpu().numpy(), ref) < tol
    ref = oracle.smoother_step(dim, k, n, x0.astype(npdt), b.astype(npdt), kappa=kap)
    x = torch.tensor(x0, dtype=dtype, device="cuda")
    tps.PatchSmoother(P).step(x, torch.tensor(b, dtype=dtype, device="cuda"))
    torch.cuda.synchronize()
    assert relerr(x.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("dim,k,n", [(2, 2, 8), (3, 2, 6), (3, 3, 4)])
def test_kappa_vcycle_and_cg(cuda, oracle, dim, k, n):
    kap = kappa_field(dim, n, 3)
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    H = oracle.Hierarchy(dim, k, P.n_coarse, P.n_levels, kappa=kap)
    b = bvec(dim, n * k + 1, 4)
    ref = H.vcycle(b, precision=0, symmetric=True)
    z = P.new_vector()
    tps.MultigridSolvers(P).vmult(z, torch.tensor(b, device="cuda"), precision="fp64", symmetric=True)
    torch.cuda.synchronize()
    assert relerr(z.cpu().numpy(), ref) < 1e-11
    xr, itr, _ = H.solve_cg(b, precision=0, symmetric=True, rel_tol=1e-10)
    x, rep = tps.MultigridSolvers(P).solve_cg(torch.tensor(b, device="cuda"), precision="fp64",
                                              rel_tol=1e-10)
    # rounding can shift the count of a longer run by one
    assert rep.converged and abs(rep.iterations - itr) <= 1 + itr // 20
    assert relerr(x.cpu().numpy(), xr) < 1e-8
    x32, rep32 = tps.MultigridSolvers(P).solve_cg(torch.tensor(b, device="cuda"), precision="fp32",
                                                  rel_tol=1e-10, max_iter=400)
    assert rep32.converged and relerr(x32.cpu().numpy(), xr) < 1e-8


@pytest.mark.parametrize("dim,k,n", [(2, 3, 4), (3, 2, 4)])
def test_mass_and_cell_energy(cuda, oracle, dim, k, n):
    kap = kappa_field(dim, n, 5)
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    N1 = n * k + 1
    from gputensorproductsmoother_b200 import problems
    M1 = problems.mass_1d(k, n)
    M = M1
    for _ in range(dim - 1):
        M = np.kron(M, M1)
    rng = np.random.default_rng(6)
    f = rng.uniform(-1, 1, N1 ** dim)
    out = P.new_vector()
    P.mass_vmult(out, torch.tensor(f, device="cuda"))
    torch.cuda.synchronize()
    assert relerr(out.cpu().numpy(), M @ f) < 1e-13
    u, lam = bvec(dim, N1, 7), bvec(dim, N1, 8)
    e = P.cell_energy(torch.tensor(u, device="cuda"), torch.tensor(lam, device="cuda")).cpu().numpy()
    for c in [0, 3, n ** dim - 1]:
        ind = np.zeros(n ** dim)
        ind[c] = 1.0
        Au = oracle.laplace_vmult(dim, k, n, u, kappa=ind)
        assert abs(e[c] - lam @ Au) <= 1e-12 * max(1.0, abs(lam @ Au))
    assert abs(e.sum() - lam @ oracle.laplace_vmult(dim, k, n, u)) < 1e-11 * np.abs(e).sum()


def test_adjoint_gradients_match_finite_differences(cuda):
    """J = 0.5 ||u - u_t||^2 with A(kappa) u = M f: the adjoint gradients agree
    with central differences (h = 1e-6) to 1e-6 in random directions."""
    dim, k, n = 3, 2, 6  # coarse 3^3 cells: dense coarse solve
    rng = np.random.default_rng(9)
    kap = torch.tensor(np.exp(rng.normal(0, 0.5, n ** dim)), dtype=torch.float64, device="cuda")
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    N = P.n_dofs()
    f = torch.tensor(rng.standard_normal(N), device="cuda", requires_grad=True)
    # target = perturbed solution, so J and its derivatives have one scale and
    # central differences are not swamped by rounding of a large J
    with torch.no_grad():
        u0 = tps.autograd.solve(P, f, kap, rel_tol=1e-14)
    ut = u0 * torch.tensor(1.0 + 0.3 * rng.standard_normal(N), device="cuda")
    kv = kap.clone().requires_grad_(True)

    def J(f_, k_):
        u = tps.autograd.solve(P, f_, k_, rel_tol=1e-14)
        return 0.5 * ((u - ut) ** 2).sum()

    j = J(f, kv)
    j.backward()
    gf, gk = f.grad.detach().clone(), kv.grad.detach().clone()
    h = 1e-6
    for d in range(4):
        df = torch.tensor(rng.standard_normal(N), device="cuda")
        dk = torch.tensor(rng.standard_normal(n ** dim), device="cuda") * kap
        with torch.no_grad():
            fd_f = (J(f + h * df, kap) - J(f - h * df, kap)) / (2 * h)
            fd_k = (J(f, kap + h * dk) - J(f, kap - h * dk)) / (2 * h)
        ad_f, ad_k = (gf * df).sum(), (gk * dk).sum()
        assert abs(ad_f - fd_f) <= 1e-6 * abs(fd_f), (d, ad_f.item(), fd_f.item())
        assert abs(ad_k - fd_k) <= 1e-6 * abs(fd_k), (d, ad_k.item(), fd_k.item())


def test_adjoint_48cubed_q4(cuda):
    """The adjoint configuration itself (Q4, 48^3 cells, coarse 3^3, kappa =
    exp(N(0, 0.5^2))): forward and adjoint MG-CG converge and two random
    directions agree with central differences (h = 1e-6) to 1e-6."""
    dim, k, n = 3, 4, 48
    rng = np.random.default_rng(0)
    kap = torch.tensor(np.exp(rng.normal(0.0, 0.5, n ** dim)), device="cuda")
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    N = P.n_dofs()
    f = torch.tensor(rng.uniform(-1, 1, N), device="cuda")
    with torch.no_grad():
        u0 = tps.autograd.solve(P, f, kap, rel_tol=1e-13)
    ut = u0 * torch.tensor(1.0 + 0.3 * rng.standard_normal(N), device="cuda")

    def J(f_, k_):
        u = tps.autograd.solve(P, f_, k_, rel_tol=1e-13)
        return 0.5 * ((u - ut) ** 2).sum()

    fv, kv = f.clone().requires_grad_(True), kap.clone().requires_grad_(True)
    J(fv, kv).backward()
    h = 1e-6
    for _ in range(2):
        df = torch.tensor(rng.standard_normal(N), device="cuda")
        dk = torch.tensor(rng.standard_normal(n ** dim), device="cuda") * kap
        with torch.no_grad():
            fd_f = (J(f + h * df, kap) - J(f - h * df, kap)) / (2 * h)
            fd_k = (J(f, kap + h * dk) - J(f, kap - h * dk)) / (2 * h)
        assert abs((fv.grad * df).sum() - fd_f) <= 1e-6 * abs(fd_f)
        assert abs((kv.grad * dk).sum() - fd_k) <= 1e-6 * abs(fd_k)
    P.close()


@pytest.mark.parametrize("dim,k,n", [(3, 2, 6), (3, 4, 12)])
def test_adjoint_matches_fp64_oracle_adjoint(cuda, oracle, dim, k, n):
    """GPU adjoint gradients (autograd.PoissonSolve backward: one tps_adjoint
    call, i.e. the MG-CG adjoint solve, M lambda and the per-cell energies)
    against the FP64 oracle adjoint
    (oracle.adjoint_gradients: the oracle's MG-CG, a dense-Kronecker mass apply
    and per-cell energies restated from the definitions) on the same seeded
    kappa, f and target: u, dJ/df and dJ/dkappa within 1e-10 (max-norm,
    relative to the largest entry).  Coarse level 3^d: dense coarse solve."""
    rng = np.random.default_rng(40 + k)
    kap_h = np.exp(rng.normal(0.0, 0.5, n ** dim))
    N1 = n * k + 1
    f_h = rng.standard_normal(N1 ** dim)
    nc, nl = tps.split_cells(n)
    H = oracle.Hierarchy(dim, k, nc, nl, kappa=kap_h)
    b = oracle.zero_dirichlet(oracle.mass_vmult(dim, k, n, f_h), dim, N1)
    u0 = H.solve_cg(b, precision=0, rel_tol=1e-14, max_it=400)[0]
    ut = u0 * (1.0 + 0.3 * rng.standard_normal(N1 ** dim))
    uo, gfo, gko = oracle.adjoint_gradients(dim, k, nc, nl, kap_h, f_h, ut, rel_tol=1e-14)

    kap = torch.tensor(kap_h, device="cuda")
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    fv = torch.tensor(f_h, device="cuda", requires_grad=True)
    kv = kap.clone().requires_grad_(True)
    u = tps.autograd.solve(P, fv, kv, rel_tol=1e-14)
    (0.5 * ((u - torch.tensor(ut, device="cuda")) ** 2).sum()).backward()
    du = relerr(u.detach().cpu().numpy(), uo)
    df = relerr(fv.grad.cpu().numpy(), gfo)
    dk = relerr(kv.grad.cpu().numpy(), gko)
    assert du <= 1e-10 and df <= 1e-10 and dk <= 1e-10, (du, df, dk)
    P.close()


def test_adjoint_abi_equals_the_composition(cuda):
    """tps_adjoint is the adjoint solve of the CG driver followed by the mass
    apply and the negated per-cell energies: bit-identical to composing
    tps_solve, tps_mass_vmult and tps_cell_energy by hand; g's Dirichlet rows
    are ignored (g is not modified); dJ/dkappa may be skipped."""
    dim, k, n = 3, 3, 8
    N1 = n * k + 1
    kap = torch.tensor(kappa_field(dim, n, 21), device="cuda")
    P = tps.PoissonProblem(dim, k, n, kappa=kap)
    MG = tps.MultigridSolvers(P)
    u, _ = MG.solve_cg(torch.tensor(bvec(dim, N1, 22), device="cuda"), precision="fp64", rel_tol=1e-13)
    g = torch.tensor(np.random.default_rng(23).uniform(-1, 1, N1 ** dim), device="cuda")  # boundary rows too
    g0 = g.clone()
    df, dk, rep = MG.adjoint(u, g, precision="fp64", rel_tol=1e-13)
    assert rep.converged and torch.equal(g, g0)
    gz = torch.tensor(bvec(dim, N1, 23), device="cuda")  # the same draws, Dirichlet rows zero
    lam, rep2 = MG.solve_cg(gz, precision="fp64", rel_tol=1e-13, max_iter=400)
    assert rep2.iterations == rep.iterations
    df_ref = torch.empty_like(lam)
    P.mass_vmult(df_ref, lam)
    dk_ref = -P.cell_energy(u, lam)
    assert torch.equal(df, df_ref) and torch.equal(dk, dk_ref)
    df2, dk2, _ = MG.adjoint(u, g, precision="fp64", rel_tol=1e-13, kappa_gradient=False)
    assert dk2 is None and torch.equal(df2, df)
    P.close()


def test_adjoint_abi_rejects_bad_requests(cuda):
    from gputensorproductsmoother_b200 import _lib as L
    import ctypes
    P = tps.PoissonProblem(3, 2, 4)  # no kappa
    u = P.new_vector()
    g = P.new_vector()
    o = L.TpsSolveOpts(L.DRIVER_CG, 0, 1, 50, 1e-10, 1e-300, 1)
    rep = L.TpsReport()
    dk = torch.empty(64, dtype=torch.float64, device="cuda")
    st = L.lib().tps_adjoint(P.handle, ctypes.byref(o), u.data_ptr(), g.data_ptr(), g.data_ptr(), None,
                             ctypes.byref(rep), None)
    assert st == 1  # TPS_ERR_INVALID: dJ/df aliases g
    df = P.new_vector()
    st = L.lib().tps_adjoint(P.handle, ctypes.byref(o), u.data_ptr(), g.data_ptr(), df.data_ptr(),
                             dk.data_ptr(), ctypes.byref(rep), None)
    assert st == 1  # dJ/dkappa without kappa
    o.driver = L.DRIVER_GMRES
    st = L.lib().tps_adjoint(P.handle, ctypes.byref(o), u.data_ptr(), g.data_ptr(), df.data_ptr(), None,
                             ctypes.byref(rep), None)
    assert st == 1
    # the handle stays usable: a zero g gives zero gradients
    o.driver = L.DRIVER_CG
    st = L.lib().tps_adjoint(P.handle, ctypes.byref(o), u.data_ptr(), g.data_ptr(), df.data_ptr(), None,
                             ctypes.byref(rep), None)
    torch.cuda.synchronize()
    assert st == L.TPS_OK and df.abs().max().item() == 0.0
    P.close()
