"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liboracle.so).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.  Parity status: UNPINNED against the
reference (LuciaZhang9/GPUTensorProductSmoother cannot be built here: it needs
deal.II with CUDA+MPI, CMakeLists.txt:81-102, and ships no golden vectors).  The
oracle is pinned instead against the independent numpy/scipy fixtures in
tests/golden/ and against mathematical known answers.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def build() -> str:
    """Compile liboracle.so with the oracle's own Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_fe1d.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
        L.orc_patch_matrices.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_gen_eig.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
        L.orc_patch_eigen.argtypes = [ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.orc_gauss.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_gauss_lobatto.argtypes = [ctypes.c_int, _dp]
        for suf, ptr in (("_d", _dp), ("_f", _fp)):
            getattr(L, "orc_laplace_vmult" + suf).argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ptr, ptr, _dp]
            getattr(L, "orc_smoother_step" + suf).argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ptr, ptr,
                ctypes.c_int, ctypes.c_int, _dp]
            getattr(L, "orc_smoother_additive" + suf).argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                ctypes.c_int]
            getattr(L, "orc_prolongate_add" + suf).argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ptr, ptr]
            getattr(L, "orc_restrict_add" + suf).argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ptr, ptr]
        L.orc_hier_create.restype = ctypes.c_void_p
        L.orc_hier_create.argtypes = [ctypes.c_int] * 4 + [_dp]
        L.orc_hier_destroy.argtypes = [ctypes.c_void_p]
        L.orc_hier_set_additive.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.orc_hier_ndofs.restype = ctypes.c_long
        L.orc_hier_ndofs.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_vcycle.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_vcycle_level.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, _dp, _dp]
        L.orc_fine_vmult.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_coarse_solve.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_solve_cg.restype = ctypes.c_int
        L.orc_solve_cg.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                   ctypes.c_double, ctypes.c_int, _dp]
        L.orc_fmg.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp),
                              ctypes.POINTER(_dp), _dp]
        for suf, ptr in (("_d", _dp), ("_f", _fp)):
            getattr(L, "orc_prolongate_add_nb" + suf).argtypes = [
                ctypes.c_int, ctypes.c_int, ctypes.c_int, ptr, ptr]
        L.orc_solve_gmres.restype = ctypes.c_int
        L.orc_solve_gmres.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(_dp)
    return a.ctypes.data_as(_fp)


def _sfx(dtype):
    return "_d" if np.dtype(dtype) == np.float64 else "_f"


def fe1d(k):
    nodes = np.zeros(k + 1)
    mass = np.zeros((k + 1, k + 1))
    lap = np.zeros((k + 1, k + 1))
    prol = np.zeros((2 * k + 1, k + 1))
    assert lib().orc_fe1d(k, _p(nodes), _p(mass), _p(lap), _p(prol)) == 0
    return nodes, mass, lap, prol


def gauss(nq):
    x = np.zeros(nq)
    w = np.zeros(nq)
    lib().orc_gauss(nq, _p(x), _p(w))
    return x, w


def patch_matrices(k):
    n1 = 2 * k + 1
    pm = np.zeros((n1, n1))
    pl = np.zeros((n1, n1))
    assert lib().orc_patch_matrices(k, _p(pm), _p(pl)) == 0
    return pm, pl


def patch_eigen(k, h):
    m = 2 * k - 1
    S = np.zeros((m, m))
    lam = np.zeros(m)
    assert lib().orc_patch_eigen(k, h, _p(S), _p(lam)) == 0
    return S, lam


def ndofs(dim, k, n):
    return (n * k + 1) ** dim


def laplace_vmult(dim, k, n, src, kappa=None):
    src = np.ascontiguousarray(src)
    dst = np.zeros_like(src)
    kap = None if kappa is None else np.ascontiguousarray(kappa, dtype=np.float64)
    getattr(lib(), "orc_laplace_vmult" + _sfx(src.dtype))(dim, k, n, _p(dst), _p(src), _p(kap))
    return dst


def smoother_step(dim, k, n, x, b, omega=1.0, zero_init=False, reverse=False, kappa=None):
    """In-place coloured sweep on a copy of x; returns the new x."""
    x = np.array(x, copy=True)
    b = np.ascontiguousarray(b, dtype=x.dtype)
    kap = None if kappa is None else np.ascontiguousarray(kappa, dtype=np.float64)
    getattr(lib(), "orc_smoother_step" + _sfx(x.dtype))(
        dim, k, n, omega, _p(x), _p(b), int(zero_init), int(reverse), _p(kap))
    return x


def smoother_additive(dim, k, n, x, b, omega, zero_init=False):
    """Additive vertex-patch Schwarz step on a copy of x (every patch's residual
    from the old x, solves summed, x += omega * sum); returns the new x."""
    x = np.array(x, copy=True)
    b = np.ascontiguousarray(b, dtype=x.dtype)
    getattr(lib(), "orc_smoother_additive" + _sfx(x.dtype))(dim, k, n, omega, _p(x), _p(b), int(zero_init))
    return x


def prolongate_add(dim, k, nc, fine, coarse):
    fine = np.array(fine, copy=True)
    coarse = np.ascontiguousarray(coarse, dtype=fine.dtype)
    getattr(lib(), "orc_prolongate_add" + _sfx(fine.dtype))(dim, k, nc, _p(fine), _p(coarse))
    return fine


def restrict_add(dim, k, nc, coarse, fine):
    coarse = np.array(coarse, copy=True)
    fine = np.ascontiguousarray(fine, dtype=coarse.dtype)
    getattr(lib(), "orc_restrict_add" + _sfx(coarse.dtype))(dim, k, nc, _p(coarse), _p(fine))
    return coarse


class Hierarchy:
    """Geometric MG hierarchy of n_coarse * 2^l cells per direction, l < n_levels."""

    def __init__(self, dim, k, n_coarse, n_levels, kappa=None):
        self.dim, self.k, self.n_coarse, self.n_levels = dim, k, n_coarse, n_levels
        self._kappa = None if kappa is None else np.ascontiguousarray(kappa, dtype=np.float64)
        self.h = lib().orc_hier_create(dim, k, n_coarse, n_levels, _p(self._kappa))
        if not self.h:
            raise ValueError("invalid hierarchy parameters")
        self.N = lib().orc_hier_ndofs(self.h, n_levels - 1)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_hier_destroy(self.h)
            self.h = None

    def ndofs(self, level):
        return lib().orc_hier_ndofs(self.h, level)

    def vmult(self, src):
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros_like(src)
        lib().orc_fine_vmult(self.h, _p(dst), _p(src))
        return dst

    def set_additive(self, omega):
        """Smooth levels >= 1 of later V-cycles with the additive step (damping
        omega); omega None restores the coloured sweep."""
        lib().orc_hier_set_additive(self.h, 0 if omega is None else 1, 0.0 if omega is None else omega)

    def vcycle(self, src, precision=0, symmetric=False, level=None):
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros_like(src)
        lvl = self.n_levels - 1 if level is None else level
        lib().orc_vcycle_level(self.h, precision, int(symmetric), lvl, _p(dst), _p(src))
        return dst

    def coarse_solve(self, src):
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros_like(src)
        lib().orc_coarse_solve(self.h, _p(dst), _p(src))
        return dst

    def solve_cg(self, b, precision=0, symmetric=True, rel_tol=1e-10, max_it=100, x0=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        hist = np.zeros(max_it + 1)
        it = lib().orc_solve_cg(self.h, precision, int(symmetric), _p(b), _p(x), rel_tol, max_it,
                                _p(hist))
        return x, it, hist[: it + 1]

    def fmg(self, rhs_levels, bnd_levels=None, precision=1, n_cycles=1):
        """Full multigrid pass (MultigridSolvers::solve): rhs_levels[l] per level,
        bnd_levels[l] Dirichlet data (boundary entries used) or None."""
        L = self.n_levels
        rh = [np.ascontiguousarray(r, dtype=np.float64) for r in rhs_levels]
        rp = (_dp * L)(*[_p(r) for r in rh])
        bp = None
        if bnd_levels is not None:
            bd = [np.ascontiguousarray(b, dtype=np.float64) for b in bnd_levels]
            bp = (_dp * L)(*[_p(b) for b in bd])
        x = np.zeros_like(rh[-1])
        lib().orc_fmg(self.h, precision, n_cycles, rp, bp, _p(x))
        return x

    def solve_gmres(self, b, precision=2, reduce=1e-9, abs_tol=1e-16, max_it=20, basis=28):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        hist = np.zeros(max_it + 1)
        it = lib().orc_solve_gmres(self.h, precision, _p(b), _p(x), reduce, abs_tol, max_it, basis,
                                   _p(hist))
        return x, it, hist[: it + 1]


# ---- adjoint of the variable-coefficient solve (no reference counterpart) ----
# Restated from the definitions, as the FP64 reference the GPU adjoint is
# checked against: A(kappa) = sum_c kappa_c A_c (cell stiffness of Q_k with
# QGauss(k+1), h = 1/n per direction), M = the global FE mass matrix, Dirichlet
# rows as identity / zero right-hand side (include/laplace_operator.cuh:33-65,
# 86-101 is the kappa = 1 operator).
#   forward  A(kappa) u = Z M f            (Z zeroes the Dirichlet rows)
#   adjoint  A(kappa) lam = Z dJ/du
#   dJ/df = M lam,   dJ/dkappa_c = -lam_c^T A_c u_c


def _mass_global_1d(k, n):
    _, mass, _, _ = fe1d(k)
    N1 = n * k + 1
    M = np.zeros((N1, N1))
    for c in range(n):
        M[c * k:c * k + k + 1, c * k:c * k + k + 1] += mass / n
    return M


def _apply_kron(v, dim, mats):
    """(mats[dim-1] x ... x mats[0]) v for the lexicographic (x fastest) vector v."""
    N1 = mats[0].shape[1]
    w = np.asarray(v, dtype=np.float64).reshape((N1,) * dim)
    for d in range(dim):
        ax = dim - 1 - d  # axis of direction d (x is the last axis)
        w = np.moveaxis(np.tensordot(mats[d], w, axes=([1], [ax])), 0, ax)
    return w.reshape(-1)


def zero_dirichlet(v, dim, N1):
    w = np.array(v, dtype=np.float64, copy=True).reshape((N1,) * dim)
    for ax in range(dim):
        sl = [slice(None)] * dim
        sl[ax] = 0
        w[tuple(sl)] = 0.0
        sl[ax] = -1
        w[tuple(sl)] = 0.0
    return w.reshape(-1)


def mass_vmult(dim, k, n, f):
    """Global FE mass matrix times the nodal vector f (all rows)."""
    M = _mass_global_1d(k, n)
    return _apply_kron(f, dim, [M] * dim)


def _cell_blocks(v, dim, k, n):
    """Cell-local values: array [c_z, c_y, c_x, i_z, i_y, i_x] (3D; [c_y, c_x,
    i_y, i_x] in 2D) of v at DoF (c k + i) per direction."""
    N1 = n * k + 1
    w = np.asarray(v, dtype=np.float64).reshape((N1,) * dim)
    idx = np.arange(n)[:, None] * k + np.arange(k + 1)[None, :]  # (n, k+1)
    if dim == 2:
        return w[idx[:, None, :, None], idx[None, :, None, :]]  # [cy, cx, iy, ix]
    return w[idx[:, None, None, :, None, None], idx[None, :, None, None, :, None],
             idx[None, None, :, None, None, :]]


def cell_energy(dim, k, n, u, lam):
    """e_c = lam_c^T A_c u_c with the unit-coefficient cell stiffness A_c
    (h^(d-2) times the Kronecker sum of the reference 1D matrices); cells
    lexicographic (x fastest)."""
    _, Mr, Lr, _ = fe1d(k)
    U = _cell_blocks(u, dim, k, n)
    Lm = _cell_blocks(lam, dim, k, n)
    h = 1.0 / n
    if dim == 2:
        AU = np.einsum("ab,cd,yxbd->yxac", Lr, Mr, U) + np.einsum("ab,cd,yxbd->yxac", Mr, Lr, U)
        e = np.einsum("yxac,yxac->yx", Lm, AU)
    else:
        AU = (np.einsum("ab,cd,ef,zyxbdf->zyxace", Lr, Mr, Mr, U) +
              np.einsum("ab,cd,ef,zyxbdf->zyxace", Mr, Lr, Mr, U) +
              np.einsum("ab,cd,ef,zyxbdf->zyxace", Mr, Mr, Lr, U))
        e = np.einsum("zyxace,zyxace->zyx", Lm, AU)
    return h ** (dim - 2) * e.reshape(-1)


def adjoint_gradients(dim, k, n_coarse, n_levels, kappa, f, u_target, rel_tol=1e-13):
    """FP64 oracle of the adjoint gradients of J = 0.5 ||u - u_target||^2 with
    A(kappa) u = Z M f: returns (u, dJ/df, dJ/dkappa).  Both solves are the
    oracle's MG-CG with the FP64 V-cycle."""
    n = n_coarse * (1 << (n_levels - 1))
    N1 = n * k + 1
    H = Hierarchy(dim, k, n_coarse, n_levels, kappa=kappa)
    b = zero_dirichlet(mass_vmult(dim, k, n, f), dim, N1)
    u, _, _ = H.solve_cg(b, precision=0, symmetric=True, rel_tol=rel_tol, max_it=400)
    g = zero_dirichlet(u - np.asarray(u_target, dtype=np.float64), dim, N1)
    lam, _, _ = H.solve_cg(g, precision=0, symmetric=True, rel_tol=rel_tol, max_it=400)
    lam = zero_dirichlet(lam, dim, N1)
    return u, mass_vmult(dim, k, n, lam), -cell_energy(dim, k, n, u, lam)


# ---- right-hand-side assembly (include/laplace_operator.cuh:118-181) ----------
# b_i = sum over cells and QGauss(k+1) points of f(x_q) phi_i(x_q) JxW_q with
# f given at the points (cells lexicographic x fastest, then the points of a
# cell lexicographic x fastest), Dirichlet rows zero.  Restated with numpy from
# the definitions: Lagrange basis on the Gauss-Lobatto nodes, Gauss rule on [0,1].


def _shape_at_gauss(k):
    nodes = gauss_lobatto_nodes(k)
    xq, wq = gauss(k + 1)
    V = np.ones((k + 1, k + 1))
    for i, xi in enumerate(nodes):
        for m, xm in enumerate(nodes):
            if m != i:
                V[:, i] *= (xq - xm) / (xi - xm)
    return V, wq


def gauss_lobatto_nodes(k):
    nodes, _, _, _ = fe1d(k)
    return nodes


def assemble_rhs(dim, k, n, fq):
    V, wq = _shape_at_gauss(k)
    W = V * wq[:, None]  # [q][i] = w_q phi_i(x_q)
    N1 = n * k + 1
    np1 = k + 1
    h = 1.0 / n
    f = np.asarray(fq, dtype=np.float64).reshape((n,) * dim + (np1,) * dim)
    b = np.zeros((N1,) * dim)
    if dim == 2:
        loc = np.einsum("qi,pj,yxpq->yxji", W, W, f) * h ** 2  # [cy, cx, iy, ix]
        for iy in range(np1):
            for ix in range(np1):
                b[iy:iy + n * k:k, ix:ix + n * k:k] += loc[:, :, iy, ix]
    else:
        loc = np.einsum("qi,pj,rl,zyxrpq->zyxlji", W, W, W, f) * h ** 3
        for iz in range(np1):
            for iy in range(np1):
                for ix in range(np1):
                    b[iz:iz + n * k:k, iy:iy + n * k:k, ix:ix + n * k:k] += loc[:, :, :, iz, iy, ix]
    return zero_dirichlet(b.reshape(-1), dim, N1)
