"""Host-side mirror of the reference's operator API for the vertex-patch
Schwarz MG path, over the C ABI of include/tps.h.

Reference classes mirrored here (same names, argument meaning and error
behaviour -- errors raise, nothing is swallowed):

* ``LaplaceOperator``  -- include/laplace_operator.cuh:80-201 (vmult/Tvmult)
* ``PatchSmoother``    -- include/patch_smoother.cuh:91-351 (vmult/step)
* ``MGTransferCUDA``   -- include/cuda_mg_transfer.cuh:57-213
  (prolongate, prolongate_and_add, restrict_and_add)
* ``MultigridSolvers`` -- include/solver.cuh:1541-2210 (vmult, solve_gmres,
  plus the MG-preconditioned CG driver)

Vectors are torch CUDA tensors (float64 or float32, contiguous, one entry per
DoF of the level, lexicographic x-fastest numbering).  torch only provides
device memory and the current stream; every operation runs in libtps.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from . import _lib as L

_DTYPES = {torch.float64: L.TPS_F64, torch.float32: L.TPS_F32}
_PRECISIONS = {"fp64": L.VCYCLE_F64, "fp32": L.VCYCLE_F32, "fp64_rounded": L.VCYCLE_F64_ROUNDED,
               "tf32": L.VCYCLE_TF32, "tf32x3": L.VCYCLE_TF32X3}


def split_cells(n_cells: int) -> tuple[int, int]:
    """n_cells = n_coarse * 2^(n_levels-1) with the smallest n_coarse >= 2."""
    if n_cells < 2:
        raise ValueError("at least 2 cells per direction are required")
    n, levels = n_cells, 1
    while n % 2 == 0 and n // 2 >= 2:
        n //= 2
        levels += 1
    return n, levels


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class PoissonProblem:
    """Uniform Q_k discretisation of -div(grad u) = f on the unit square/cube
    with homogeneous Dirichlet data and its geometric MG hierarchy (replaces
    the Triangulation/DoFHandler set-up of apps/poisson.cu:152-181 and the
    level set-up of MultigridSolvers, include/solver.cuh:1545-1744)."""

    def __init__(self, dim: int, degree: int, n_cells: int, relaxation: float = 1.0,
                 n_coarse: int | None = None, device: int | None = None, kappa=None):
        if n_coarse is None:
            n_coarse, n_levels = split_cells(n_cells)
        else:
            q, n_levels = n_cells // n_coarse, 1
            if q * n_coarse != n_cells or q & (q - 1):
                raise ValueError("n_cells must be n_coarse * 2^l")
            while q > 1:
                q //= 2
                n_levels += 1
        self.dim, self.degree, self.n_cells = dim, degree, n_cells
        self.n_coarse, self.n_levels = n_coarse, n_levels
        self.device = torch.cuda.current_device() if device is None else device
        self.has_kappa = kappa is not None
        kap = None
        if kappa is not None:
            self._kappa_host = self._kappa_array(kappa)
            kap = self._kappa_host.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        pb = L.TpsProblem(dim, degree, n_coarse, n_levels, relaxation, kap, self.device)
        h = ctypes.c_void_p()
        L.check(L.lib().tps_create(ctypes.byref(pb), ctypes.byref(h)), None)
        self._h = h

    def n_cells_total(self) -> int:
        return self.n_cells ** self.dim

    def _kappa_array(self, kappa):
        import numpy as np
        if isinstance(kappa, torch.Tensor):
            kappa = kappa.detach().to("cpu", torch.float64).numpy()
        a = np.ascontiguousarray(kappa, dtype=np.float64).ravel()
        if a.size != self.n_cells ** self.dim:
            raise ValueError(f"kappa needs {self.n_cells ** self.dim} per-cell values, got {a.size}")
        return a

    def set_kappa(self, kappa, rebuild_coarse: bool = True) -> None:
        """Replace the per-cell coefficient (handle created with a kappa)."""
        self._kappa_host = self._kappa_array(kappa)
        L.check(L.lib().tps_set_kappa(self.handle, self._kappa_host.ctypes.data, int(rebuild_coarse)),
                self.handle)

    def time_smoother(self, level: int | None = None, dtype: str = "fp32", sweeps: int = 20) -> float:
        """Milliseconds per coloured sweep on the level's V-cycle work vectors
        (CUDA events on the current stream); dtype "fp64", "fp32" or "tf32"
        (tensor-core patch solves)."""
        codes = {"fp64": L.TPS_F64, "fp32": L.TPS_F32, "tf32": L.TPS_TF32, "tf32x3": L.TPS_TF32X3}
        ms = ctypes.c_double()
        lv = self.n_levels - 1 if level is None else level
        L.check(L.lib().tps_time_smoother(self.handle, lv, codes[dtype], sweeps, ctypes.byref(ms), _stream()),
                self.handle)
        return ms.value

    def autotune(self, dtype: str = "fp32") -> list[int]:
        """Time the 3D smoother's kernel variants and the operator's tile
        depths on every level and keep the fastest; returns the chosen patches
        per batch per level (-1: the one-warp-per-patch kernel, -2: two
        patches per warp in packed FP32)."""
        out = (ctypes.c_int * self.n_levels)()
        L.check(L.lib().tps_autotune(self.handle, {"fp64": L.TPS_F64, "fp32": L.TPS_F32}[dtype], out),
                self.handle)
        return list(out)

    def operator_layers(self, level: int | None = None, dtype: str = "fp32") -> int:
        """Cell layers per CTA of the 3D operator on a level (set by autotune;
        0 = the library's rule)."""
        lv = self.n_levels - 1 if level is None else level
        out = ctypes.c_int()
        L.check(L.lib().tps_get_operator_layers(self.handle, {"fp64": L.TPS_F64, "fp32": L.TPS_F32}[dtype], lv,
                                                ctypes.byref(out)), self.handle)
        return out.value

    def set_operator_layers(self, layers: int, dtype: str = "fp32", level: int | None = None) -> None:
        """Cell layers per CTA of the 3D operator on one level (all if None);
        0 = the library's rule."""
        code = {"fp64": L.TPS_F64, "fp32": L.TPS_F32}[dtype]
        for lv in range(self.n_levels) if level is None else [level]:
            L.check(L.lib().tps_set_operator_layers(self.handle, code, lv, layers), self.handle)

    def smoother_variants(self, dtype: str = "fp32") -> list[int]:
        """Patches per batch of each compiled 3D smoother variant (index =
        variant; -1: one warp per patch; -2: two patches per warp in packed
        FP32; 0 in 2D)."""
        out = (ctypes.c_int * L.SMOOTHER_VARIANTS)()
        L.check(L.lib().tps_smoother_variants(self.handle, {"fp64": L.TPS_F64, "fp32": L.TPS_F32}[dtype], out),
                self.handle)
        return list(out)

    def set_smoother_kind(self, kind: str = "fused", damping: float = 0.0) -> None:
        """Smoothing of the V-cycle's levels >= 1: "fused" (the reference's
        coloured multiplicative sweep, the default) or "additive" (the
        additive vertex-patch Schwarz step, damping in [0, 2/2^dim), 0 selects
        1/2^dim).  The coarse solve is unchanged."""
        code = {"fused": L.SMOOTHER_FUSED, "additive": L.SMOOTHER_ADDITIVE}[kind]
        L.check(L.lib().tps_set_smoother_kind(self.handle, code, float(damping)), self.handle)

    def smoother_variant(self, level: int | None = None, dtype: str = "fp32") -> int:
        """The 3D smoother variant the level's sweeps use now (set, autotuned
        or the library default)."""
        v = ctypes.c_int()
        lv = self.n_levels - 1 if level is None else level
        L.check(L.lib().tps_get_smoother_variant(self.handle, {"fp64": L.TPS_F64, "fp32": L.TPS_F32}[dtype], lv,
                                                 ctypes.byref(v)), self.handle)
        return v.value

    def set_smoother_variant(self, variant: int, dtype: str = "fp32", level: int | None = None) -> None:
        """Use smoother variant `variant` on one level (all levels if None)."""
        code = {"fp64": L.TPS_F64, "fp32": L.TPS_F32}[dtype]
        for lv in range(self.n_levels) if level is None else [level]:
            L.check(L.lib().tps_set_smoother_variant(self.handle, code, lv, variant), self.handle)

    def mass_vmult(self, dst: torch.Tensor, src: torch.Tensor) -> None:
        """dst = M src (finest level, all rows, FP64)."""
        lvl = self.n_levels - 1
        self._check_vec(dst, lvl, torch.float64)
        self._check_vec(src, lvl, torch.float64)
        L.check(L.lib().tps_mass_vmult(self.handle, dst.data_ptr(), src.data_ptr(), _stream()),
                self.handle)

    def quadrature_points(self, level: int | None = None):
        """Coordinates of the QGauss(k+1) points of every cell of the level, in
        the order tps_assemble_rhs expects: cells lexicographic (x fastest),
        then the points of a cell lexicographic (x fastest).  Returns dim
        float64 CUDA tensors (x, y[, z]) of shape (cells, (k+1)^dim)."""
        import numpy as np
        lv = self.n_levels - 1 if level is None else level
        n, k, d = self.cells(lv), self.degree, self.dim
        xq = 0.5 * (np.polynomial.legendre.leggauss(k + 1)[0] + 1.0)
        dev = torch.device("cuda", self.device)
        c = torch.arange(n, dtype=torch.float64, device=dev)
        q = torch.tensor(xq, dtype=torch.float64, device=dev)
        t = (c[:, None] + q[None, :]) / n  # (cell, point) per direction
        if d == 2:
            xs = t[None, :, None, :].expand(n, n, k + 1, k + 1)
            ys = t[:, None, :, None].expand(n, n, k + 1, k + 1)
            return xs.reshape(n * n, -1), ys.reshape(n * n, -1)
        xs = t[None, None, :, None, None, :].expand(n, n, n, k + 1, k + 1, k + 1)
        ys = t[None, :, None, None, :, None].expand(n, n, n, k + 1, k + 1, k + 1)
        zs = t[:, None, None, :, None, None].expand(n, n, n, k + 1, k + 1, k + 1)
        return xs.reshape(n ** 3, -1), ys.reshape(n ** 3, -1), zs.reshape(n ** 3, -1)

    def assemble_rhs(self, f, level: int | None = None) -> torch.Tensor:
        """b_i = sum over cells and QGauss(k+1) points of f(x_q) phi_i(x_q) JxW_q
        on the device (tps_assemble_rhs; the right-hand-side loop of
        LaplaceOperator::compute_residual, include/laplace_operator.cuh:118-181),
        Dirichlet rows zero.  f: a callable of the point coordinates
        (quadrature_points) returning a tensor of the same shape, or the values
        at the points themselves."""
        lv = self.n_levels - 1 if level is None else level
        fq = f if isinstance(f, torch.Tensor) else f(*self.quadrature_points(lv))
        fq = fq.to(torch.float64).contiguous()
        nq = (self.degree + 1) ** self.dim * self.cells(lv) ** self.dim
        if not fq.is_cuda or fq.numel() != nq:
            raise ValueError(f"f needs {nq} values on the device (cells x Gauss points)")
        b = self.new_vector(lv)
        L.check(L.lib().tps_assemble_rhs(self.handle, lv, fq.data_ptr(), b.data_ptr(), _stream()), self.handle)
        return b

    def cell_energy(self, u: torch.Tensor, lam: torch.Tensor) -> torch.Tensor:
        """Per finest-level cell: lambda_c^T A_cell u_c (FP64)."""
        lvl = self.n_levels - 1
        self._check_vec(u, lvl, torch.float64)
        self._check_vec(lam, lvl, torch.float64)
        e = torch.empty(self.n_cells ** self.dim, dtype=torch.float64, device=u.device)
        L.check(L.lib().tps_cell_energy(self.handle, u.data_ptr(), lam.data_ptr(), e.data_ptr(),
                                        _stream()), self.handle)
        return e

    def check_device(self) -> None:
        """Synchronizes the device and raises TpsError(TPS_ERR_TIMEOUT) when a
        bounded device wait of an earlier level call ran out (the flag is
        cleared by the check).  The solvers check it themselves."""
        L.check(L.lib().tps_device_status(self.handle), self.handle)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().tps_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("problem has been closed")
        return self._h

    def n_dofs(self, level: int | None = None) -> int:
        lvl = self.n_levels - 1 if level is None else level
        n = ctypes.c_int64()
        c = ctypes.c_int()
        L.check(L.lib().tps_level_info(self.handle, lvl, ctypes.byref(n), ctypes.byref(c)),
                self.handle)
        return n.value

    def cells(self, level: int | None = None) -> int:
        lvl = self.n_levels - 1 if level is None else level
        return self.n_coarse << lvl

    def new_vector(self, level: int | None = None, dtype=torch.float64) -> torch.Tensor:
        """LaplaceOperator::initialize_dof_vector equivalent."""
        return torch.zeros(self.n_dofs(level), dtype=dtype, device=f"cuda:{self.device}")

    def _check_vec(self, v: torch.Tensor, level: int, dtype=None) -> int:
        if not isinstance(v, torch.Tensor) or not v.is_cuda:
            raise TypeError("vectors must be CUDA tensors")
        if not v.is_contiguous():
            raise ValueError("vectors must be contiguous")
        if v.numel() != self.n_dofs(level):
            raise ValueError(f"vector has {v.numel()} entries, level {level} has {self.n_dofs(level)}")
        if v.dtype not in _DTYPES or (dtype is not None and v.dtype != dtype):
            raise TypeError(f"unsupported dtype {v.dtype}")
        return _DTYPES[v.dtype]


class LaplaceOperator:
    """LaplaceOperator<dim, k, Number>::vmult on one level: dst = A src on the
    interior rows, dst = src on the Dirichlet rows."""

    def __init__(self, problem: PoissonProblem, level: int | None = None):
        self.problem = problem
        self.level = problem.n_levels - 1 if level is None else level

    def vmult(self, dst: torch.Tensor, src: torch.Tensor) -> None:
        p = self.problem
        dt = p._check_vec(dst, self.level)
        p._check_vec(src, self.level, dst.dtype)
        L.check(L.lib().tps_laplace_vmult(p.handle, self.level, dt, dst.data_ptr(), src.data_ptr(),
                                          _stream()), p.handle)

    Tvmult = vmult

    def initialize_dof_vector(self, dtype=torch.float64) -> torch.Tensor:
        return self.problem.new_vector(self.level, dtype)


class PatchSmoother:
    """PatchSmoother (PreconditionRelaxation over the coloured vertex-patch
    sweep): vmult zeroes dst and sweeps once, step sweeps once in place.
    tensor_cores=True (or "tf32") runs the 3D patch solves of FP32 vectors on
    the tensor cores (TF32 operands, FP32 accumulation); "tf32x3" forms every
    product from a three-term TF32 split (about FP32 accuracy, degree 4 only).
    variant selects the
    reference's SmootherVariant (include/patch_base.cuh:28-90): "fused" (the
    default kernels), or the separate-kernel cross-checks "separate" (patch
    residual kernel + fast-diagonalisation kernel), "global" (level operator
    residual + fast diagonalisation) and "exact" (patch residual + dense
    inverse of the interior patch matrix); "additive" is the additive
    vertex-patch Schwarz step (no reference counterpart), damped by the
    problem's additive damping (PoissonProblem.set_smoother_kind)."""

    VARIANTS = {"fused": L.SMOOTHER_FUSED, "separate": L.SMOOTHER_SEPARATE, "global": L.SMOOTHER_GLOBAL,
                "exact": L.SMOOTHER_EXACT, "additive": L.SMOOTHER_ADDITIVE}

    def __init__(self, problem: PoissonProblem, level: int | None = None, tensor_cores: bool = False,
                 variant: str = "fused"):
        self.problem = problem
        self.level = problem.n_levels - 1 if level is None else level
        if tensor_cores not in (False, True, "tf32", "tf32x3"):
            raise ValueError(f"tensor_cores must be False, True, 'tf32' or 'tf32x3', not {tensor_cores!r}")
        self.tensor_cores = "tf32" if tensor_cores is True else tensor_cores
        if variant not in self.VARIANTS:
            raise ValueError(f"unknown smoother variant {variant!r}")
        if tensor_cores and variant != "fused":
            raise ValueError("the tensor-core smoother is a fused kernel")
        self.variant = variant

    def _sweep(self, dst, src, zero_init: bool, reverse: bool):
        p = self.problem
        dt = p._check_vec(dst, self.level)
        p._check_vec(src, self.level, dst.dtype)
        if self.tensor_cores:
            if dst.dtype != torch.float32:
                raise TypeError("the tensor-core smoother works on float32 vectors")
            dt = L.TPS_TF32X3 if self.tensor_cores == "tf32x3" else L.TPS_TF32
        if self.variant == "fused":
            L.check(L.lib().tps_smoother_step(p.handle, self.level, dt, dst.data_ptr(), src.data_ptr(),
                                              int(zero_init), int(reverse), _stream()), p.handle)
        else:
            L.check(L.lib().tps_smoother_step_variant(p.handle, self.level, dt, dst.data_ptr(), src.data_ptr(),
                                                      int(zero_init), int(reverse), self.VARIANTS[self.variant],
                                                      _stream()), p.handle)

    def vmult(self, dst: torch.Tensor, src: torch.Tensor, reverse: bool = False) -> None:
        self._sweep(dst, src, True, reverse)

    def step(self, dst: torch.Tensor, src: torch.Tensor, reverse: bool = False) -> None:
        self._sweep(dst, src, False, reverse)

    def Tvmult(self, dst, src):  # include/patch_smoother.cuh:55-67: no-op in the reference
        pass

    def Tstep(self, dst, src):
        pass


class MGTransferCUDA:
    """Geometric transfer between consecutive levels (to_level / from_level is
    the finer one)."""

    def __init__(self, problem: PoissonProblem):
        self.problem = problem

    def prolongate(self, to_level: int, dst: torch.Tensor, src: torch.Tensor) -> None:
        dst.zero_()
        self.prolongate_and_add(to_level, dst, src)

    def prolongate_and_add(self, to_level: int, dst: torch.Tensor, src: torch.Tensor) -> None:
        p = self.problem
        dt = p._check_vec(dst, to_level)
        p._check_vec(src, to_level - 1, dst.dtype)
        L.check(L.lib().tps_prolongate_add(p.handle, to_level, dt, dst.data_ptr(), src.data_ptr(),
                                           _stream()), p.handle)

    def restrict_and_add(self, from_level: int, dst: torch.Tensor, src: torch.Tensor) -> None:
        p = self.problem
        dt = p._check_vec(dst, from_level - 1)
        p._check_vec(src, from_level, dst.dtype)
        L.check(L.lib().tps_restrict_add(p.handle, from_level, dt, dst.data_ptr(), src.data_ptr(),
                                         _stream()), p.handle)


@dataclass
class SolveReport:
    iterations: int
    converged: bool
    initial_residual: float
    final_residual: float
    history: list = field(default_factory=list)
    time_ms: float = 0.0


def _report(r: L.TpsReport) -> SolveReport:
    n = min(r.iterations + 1, L.MAX_HISTORY)
    return SolveReport(r.iterations, bool(r.converged), r.initial_residual, r.final_residual,
                       [r.history[i] for i in range(n)], r.time_ms)


class MultigridSolvers:
    """MG-preconditioned Krylov solves on the finest level (FP64 outer
    iteration, V-cycle in FP64, FP32, or FP64 with FP32-rounded input)."""

    def __init__(self, problem: PoissonProblem):
        self.problem = problem

    def vmult(self, dst: torch.Tensor, src: torch.Tensor, precision: str = "fp32",
              symmetric: bool = False) -> None:
        """One V-cycle applied to src (MultigridSolvers::vmult)."""
        p = self.problem
        lvl = p.n_levels - 1
        p._check_vec(dst, lvl, torch.float64)
        p._check_vec(src, lvl, torch.float64)
        L.check(L.lib().tps_vcycle(p.handle, _PRECISIONS[precision], int(symmetric), dst.data_ptr(),
                                   src.data_ptr(), _stream()), p.handle)

    def _solve(self, driver, b, x, precision, symmetric, max_iter, rel_tol, abs_tol, use_graph,
               raise_on_fail):
        p = self.problem
        lvl = p.n_levels - 1
        p._check_vec(b, lvl, torch.float64)
        if x is None:
            x = torch.zeros_like(b)
        p._check_vec(x, lvl, torch.float64)
        o = L.TpsSolveOpts(driver, _PRECISIONS[precision], int(symmetric), max_iter, rel_tol,
                           abs_tol, int(use_graph))
        rep = L.TpsReport()
        st = L.lib().tps_solve(p.handle, ctypes.byref(o), b.data_ptr(), x.data_ptr(),
                               ctypes.byref(rep), _stream())
        if st != L.TPS_OK and (raise_on_fail or st != 4):
            L.check(st, p.handle)
        return x, _report(rep)

    def solve_fmg(self, rhs_levels, bnd_levels=None, precision: str = "fp32", n_cycles: int = 1):
        """MultigridSolvers::solve: one full-multigrid pass.  rhs_levels[l]: the
        right-hand side of level l (float64 CUDA tensors, lifting of the
        Dirichlet data included); bnd_levels[l] (optional): Dirichlet values on
        the boundary DoFs of level l.  Returns (x, SolveReport)."""
        p = self.problem
        n = p.n_levels
        if len(rhs_levels) != n or (bnd_levels is not None and len(bnd_levels) != n):
            raise ValueError(f"one vector per level ({n}) is required")
        for l in range(n):
            p._check_vec(rhs_levels[l], l, torch.float64)
            if bnd_levels is not None:
                p._check_vec(bnd_levels[l], l, torch.float64)
        x = p.new_vector()
        rp = (ctypes.c_void_p * n)(*[r.data_ptr() for r in rhs_levels])
        bp = None if bnd_levels is None else (ctypes.c_void_p * n)(*[b.data_ptr() for b in bnd_levels])
        rep = L.TpsReport()
        L.check(L.lib().tps_fmg(p.handle, _PRECISIONS[precision], n_cycles, rp, bp, x.data_ptr(),
                                ctypes.byref(rep), _stream()), p.handle)
        return x, _report(rep)

    def solve_cg(self, b: torch.Tensor, x: torch.Tensor | None = None, precision: str = "fp32",
                 symmetric: bool = True, max_iter: int = 100, rel_tol: float = 1e-10,
                 use_graph: bool = True, raise_on_fail: bool = True):
        """Flexible CG, FP64 outer iteration, to ||b - A x|| <= rel_tol ||b||."""
        return self._solve(L.DRIVER_CG, b, x, precision, symmetric, max_iter, rel_tol, 1e-300,
                           use_graph, raise_on_fail)

    def adjoint(self, u: torch.Tensor, g: torch.Tensor, precision: str = "fp64", rel_tol: float = 1e-13,
                max_iter: int = 400, kappa_gradient: bool = True, raise_on_fail: bool = True):
        """Adjoint gradients of J(u(f, kappa)) through tps_adjoint: given the
        forward solution u and g = dJ/du, solves A lambda = g (Dirichlet rows
        of g taken as zero) and returns (dJ/df = M lambda, dJ/dkappa =
        -lambda_c^T A_c u_c per cell or None, SolveReport)."""
        p = self.problem
        lv = p.n_levels - 1
        p._check_vec(u, lv, torch.float64)
        p._check_vec(g, lv, torch.float64)
        dJdf = torch.empty_like(u)
        dk = None
        if kappa_gradient and p.has_kappa:
            n = p.cells(lv)
            dk = torch.empty(n ** p.dim, dtype=torch.float64, device=u.device)
        o = L.TpsSolveOpts(L.DRIVER_CG, _PRECISIONS[precision], 1, max_iter, rel_tol, 1e-300, 1)
        rep = L.TpsReport()
        st = L.lib().tps_adjoint(p.handle, ctypes.byref(o), u.data_ptr(), g.data_ptr(), dJdf.data_ptr(),
                                 None if dk is None else dk.data_ptr(), ctypes.byref(rep), _stream())
        if st != L.TPS_OK and (raise_on_fail or st != 4):
            L.check(st, p.handle)
        return dJdf, dk, _report(rep)

    def solve_host_many(self, bs, xs=None, precision: str = "fp32", symmetric: bool = True,
                        max_iter: int = 100, rel_tol: float = 1e-10, raise_on_fail: bool = True):
        """CG solves (each from x = 0) of a sequence of HOST right-hand sides
        (contiguous CPU float64 tensors), the copies of one solve overlapped
        with its neighbours' solves (tps_solve_host_many); pinned tensors are
        needed for the overlap.  xs: output tensors (allocated pinned when
        None).  Returns (xs, list of SolveReport)."""
        p = self.problem
        n, N = len(bs), p.n_dofs()
        if n < 1:
            raise ValueError("at least one right-hand side is required")
        if xs is None:
            xs = [torch.empty(N, dtype=torch.float64).pin_memory() for _ in range(n)]
        if len(xs) != n:
            raise ValueError(f"{n} output tensors are required")
        for v in list(bs) + list(xs):
            if v.is_cuda or v.dtype != torch.float64 or not v.is_contiguous() or v.numel() != N:
                raise ValueError(f"host vectors must be contiguous CPU float64 tensors of {N} entries")
        o = L.TpsSolveOpts(L.DRIVER_CG, _PRECISIONS[precision], int(symmetric), max_iter, rel_tol, 1e-300, 1)
        reps = (L.TpsReport * n)()
        bp = (ctypes.c_void_p * n)(*[b.data_ptr() for b in bs])
        xp = (ctypes.c_void_p * n)(*[x.data_ptr() for x in xs])
        st = L.lib().tps_solve_host_many(p.handle, ctypes.byref(o), n, bp, xp, reps)
        if st != L.TPS_OK and (raise_on_fail or st != 4):
            L.check(st, p.handle)
        return xs, [_report(reps[i]) for i in range(n)]

    def solve_gmres(self, b: torch.Tensor, x: torch.Tensor | None = None,
                    precision: str = "fp64_rounded", max_iter: int = 20, reduce: float = 1e-9,
                    abs_tol: float = 1e-16, raise_on_fail: bool = False):
        """deal.II-SolverGMRES-semantics solve as in MultigridSolvers::solve_gmres
        (non-convergence is reported, not raised, like the reference)."""
        return self._solve(L.DRIVER_GMRES, b, x, precision, False, max_iter, reduce, abs_tol,
                           False, raise_on_fail)


class BatchSolver:
    """Many independent Poisson systems solved together by one CUDA graph
    launch (tps_batch_*): right-hand sides of one mesh and/or meshes of
    different sizes.  ``systems`` is a list of (dim, degree, n_cells) or
    (dim, degree, n_cells, n_coarse) tuples, one per system."""

    def __init__(self, systems, relaxation: float = 1.0, device: int | None = None):
        dev = torch.cuda.current_device() if device is None else device
        self.shapes = []
        arr = (L.TpsProblem * len(systems))()
        for i, sysdef in enumerate(systems):
            dim, degree, n_cells = sysdef[:3]
            if len(sysdef) > 3:
                n_coarse = sysdef[3]
                q, n_levels = n_cells // n_coarse, 1
                while q > 1:
                    q //= 2
                    n_levels += 1
            else:
                n_coarse, n_levels = split_cells(n_cells)
            arr[i] = L.TpsProblem(dim, degree, n_coarse, n_levels, relaxation, None, dev)
            self.shapes.append((dim, degree, n_cells))
        h = ctypes.c_void_p()
        st = L.lib().tps_batch_create(arr, len(systems), ctypes.byref(h))
        if st != L.TPS_OK:
            msg = L.lib().tps_batch_last_error(None)
            raise L.TpsError(st, msg.decode() if msg else "")
        self._h = h
        self.device = dev

    def __len__(self) -> int:
        return len(self.shapes)

    def n_dofs(self, i: int) -> int:
        dim, degree, n = self.shapes[i]
        return (n * degree + 1) ** dim

    def solve(self, rhs, x=None, precision: str = "fp32", symmetric: bool = True, max_iter: int = 100,
              rel_tol: float = 1e-10, raise_on_fail: bool = True):
        """Solves every system; rhs (and x) are lists of CUDA float64 tensors.
        Returns (x list, list of SolveReport)."""
        n = len(self.shapes)
        if len(rhs) != n:
            raise ValueError(f"{n} right-hand sides are required")
        for i, b in enumerate(rhs):
            if not (b.is_cuda and b.dtype == torch.float64 and b.is_contiguous() and b.numel() == self.n_dofs(i)):
                raise ValueError(f"rhs[{i}] must be a contiguous CUDA float64 tensor of {self.n_dofs(i)} entries")
        xs = [torch.zeros_like(b) for b in rhs] if x is None else list(x)
        bp = (ctypes.c_void_p * n)(*[b.data_ptr() for b in rhs])
        xp = (ctypes.c_void_p * n)(*[v.data_ptr() for v in xs])
        o = L.TpsSolveOpts(L.DRIVER_CG, _PRECISIONS[precision], int(symmetric), max_iter, rel_tol, 1e-300, 1)
        reps = (L.TpsReport * n)()
        st = L.lib().tps_batch_solve(self._h, ctypes.byref(o), bp, xp, reps, _stream())
        if st != L.TPS_OK and (raise_on_fail or st != 4):
            msg = L.lib().tps_batch_last_error(self._h)
            raise L.TpsError(st, msg.decode() if msg else "")
        return xs, [_report(reps[i]) for i in range(n)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            L.lib().tps_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

