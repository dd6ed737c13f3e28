"""GPU tests of failure detection: every failure is made on the host (a bad
argument, a non-finite or underflowing right-hand side, too few iterations,
an injected allocation failure) or by a bounded device wait that nothing
completes, and each must come back as its status with the handle still
usable.  Nothing here faults or hangs the GPU: the timed-out wait gives up
after ~2^20 SM cycles and its kernel returns normally."""
import ctypes

import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import _lib as L

pytestmark = pytest.mark.gpu

INVALID, ALLOC, NOT_CONVERGED, BREAKDOWN, NONFINITE, TIMEOUT = 1, 3, 4, 5, 6, 8
SHORT_WAIT = 1 << 20  # SM cycles, well under a millisecond


def interior_random(dim, N1, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, N1 ** dim) * scale
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return torch.tensor(v, device="cuda")


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def raw_solve(P, b, x, precision=L.VCYCLE_F32, driver=L.DRIVER_CG, max_iter=100, rel_tol=1e-10,
              use_graph=1):
    o = L.TpsSolveOpts(driver, precision, 1 if driver == L.DRIVER_CG else 0, max_iter, rel_tol, 1e-300,
                       use_graph)
    rep = L.TpsReport()
    st = L.lib().tps_solve(P.handle, ctypes.byref(o), b.data_ptr(), x.data_ptr(), ctypes.byref(rep), stream())
    torch.cuda.synchronize()
    return st, rep


def test_invalid_arguments_leave_the_handle_usable(cuda):
    lib = L.lib()
    P = tps.PoissonProblem(3, 2, 8)
    h, nl = P.handle, P.n_levels
    a = P.new_vector()
    c = P.new_vector()
    s = stream()
    for lvl in (-1, nl):
        assert lib.tps_laplace_vmult(h, lvl, L.TPS_F64, a.data_ptr(), c.data_ptr(), s) == INVALID
        assert lib.tps_smoother_step(h, lvl, L.TPS_F64, a.data_ptr(), c.data_ptr(), 0, 0, s) == INVALID
        assert b"out of range" in lib.tps_last_error(h)
    assert lib.tps_prolongate_add(h, 0, L.TPS_F64, a.data_ptr(), c.data_ptr(), s) == INVALID
    assert lib.tps_restrict_add(h, 0, L.TPS_F64, a.data_ptr(), c.data_ptr(), s) == INVALID
    assert lib.tps_laplace_vmult(h, nl - 1, 7, a.data_ptr(), c.data_ptr(), s) == INVALID
    assert lib.tps_laplace_vmult(h, nl - 1, L.TPS_F64, None, c.data_ptr(), s) == INVALID
    assert lib.tps_laplace_vmult(h, nl - 1, L.TPS_F64, a.data_ptr(), a.data_ptr(), s) == INVALID
    assert lib.tps_smoother_step_variant(h, nl - 1, L.TPS_F64, a.data_ptr(), c.data_ptr(), 0, 0, 9, s) == INVALID
    assert lib.tps_vcycle(h, L.VCYCLE_F32, 1, None, c.data_ptr(), s) == INVALID
    assert lib.tps_set_smoother_kind(h, L.SMOOTHER_ADDITIVE, 0.25) == INVALID  # >= 2/2^3
    assert lib.tps_selftest_wait_timeout(h, 0, s) == INVALID
    assert lib.tps_selftest_wait_timeout(h, (1 << 31) + 1, s) == INVALID
    b = interior_random(3, 17, 3)
    x = torch.zeros_like(b)
    assert raw_solve(P, b, x, max_iter=0)[0] == INVALID
    assert raw_solve(P, b, x, driver=5)[0] == INVALID
    assert raw_solve(P, b, x, precision=5)[0] == INVALID
    assert x.abs().max().item() == 0.0  # nothing ran
    st, rep = raw_solve(P, b, x)
    assert st == L.TPS_OK and rep.converged
    assert lib.tps_last_error(h) == b""
    assert lib.tps_device_status(h) == L.TPS_OK
    P.close()


@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
@pytest.mark.parametrize("driver", [L.DRIVER_CG, L.DRIVER_GMRES])
def test_nonfinite_rhs(cuda, bad, driver):
    P = tps.PoissonProblem(3, 3, 8)
    b = interior_random(3, 25, 5)
    b[25 * 25 * 12 + 25 * 12 + 12] = bad
    x = torch.zeros_like(b)
    st, rep = raw_solve(P, b, x, driver=driver, precision=L.VCYCLE_F32 if driver == L.DRIVER_CG
                        else L.VCYCLE_F64_ROUNDED)
    assert st == NONFINITE, st
    assert not rep.converged
    assert b"non-finite" in L.lib().tps_last_error(P.handle)
    # the same handle then solves a finite system
    b2 = interior_random(3, 25, 6)
    x2 = torch.zeros_like(b2)
    st, rep = raw_solve(P, b2, x2, driver=driver, precision=L.VCYCLE_F32 if driver == L.DRIVER_CG
                        else L.VCYCLE_F64_ROUNDED, max_iter=100, rel_tol=1e-9)
    assert st == L.TPS_OK and rep.converged
    P.close()


@pytest.mark.parametrize("driver", [L.DRIVER_CG, L.DRIVER_GMRES])
def test_max_iteration_exhaustion(cuda, driver):
    P = tps.PoissonProblem(3, 3, 8)
    b = interior_random(3, 25, 7)
    x = torch.zeros_like(b)
    st, rep = raw_solve(P, b, x, driver=driver, max_iter=1, rel_tol=1e-14,
                        precision=L.VCYCLE_F32 if driver == L.DRIVER_CG else L.VCYCLE_F64_ROUNDED)
    assert st == NOT_CONVERGED
    assert rep.iterations == 1 and not rep.converged
    assert rep.history[0] == 1.0 and 0.0 < rep.history[1] < 1.0
    assert x.abs().max().item() > 0.0  # the iterate of the one step is returned
    assert b"max_iter" in L.lib().tps_last_error(P.handle)
    # the Python drivers raise, unless told to report
    with pytest.raises(tps.TpsError) as ei:
        tps.MultigridSolvers(P).solve_cg(b, max_iter=1, rel_tol=1e-14)
    assert ei.value.status == NOT_CONVERGED
    _, r = tps.MultigridSolvers(P).solve_cg(b, max_iter=1, rel_tol=1e-14, raise_on_fail=False)
    assert r.iterations == 1 and not r.converged
    P.close()


@pytest.mark.parametrize("dim,k,n", [(3, 3, 8), (2, 4, 16)])
def test_cg_breakdown_on_underflowing_fp32_residual(cuda, dim, k, n):
    """A residual of size ~1e-50 rounds to zero in the FP32 V-cycle: the
    preconditioned direction p is zero, p^T A p = 0, and CG stops with
    TPS_ERR_BREAKDOWN instead of dividing by zero.  The FP64 V-cycle solves
    the same system."""
    P = tps.PoissonProblem(dim, k, n)
    b = interior_random(dim, n * k + 1, 9, scale=1e-50)
    x = torch.zeros_like(b)
    st, rep = raw_solve(P, b, x, precision=L.VCYCLE_F32)
    assert st == BREAKDOWN, st
    assert not rep.converged and rep.iterations == 1
    assert b"breakdown" in L.lib().tps_last_error(P.handle)
    assert x.abs().max().item() == 0.0  # alpha = 0: the iterate is untouched
    x64 = torch.zeros_like(b)
    st, rep = raw_solve(P, b, x64, precision=L.VCYCLE_F64)
    assert st == L.TPS_OK and rep.converged and rep.final_residual <= 1e-10
    P.close()


def test_batch_reports_per_system_failures(cuda):
    B = tps.BatchSolver([(3, 3, 8), (3, 3, 8), (3, 2, 6)])
    rhs = [interior_random(3, 25, 11), interior_random(3, 25, 12), interior_random(3, 13, 13)]
    rhs[1][25 * 25 * 12 + 25 * 12 + 12] = float("nan")
    with pytest.raises(tps.TpsError) as ei:
        B.solve(rhs, precision="fp32", rel_tol=1e-10)
    assert ei.value.status == NONFINITE
    rhs[1] = interior_random(3, 25, 12)
    xs, reps = B.solve(rhs, precision="fp32", rel_tol=1e-10)
    assert all(r.converged for r in reps)
    B.close()


def test_injected_allocation_failures(cuda):
    """Fail the n-th device allocation of a solve for n = 1, 2, ... until the
    solve needs fewer: every failed call returns TPS_ERR_ALLOC, the handle
    keeps working, and the first successful solve equals the solve of a
    handle that never failed, bit for bit."""
    lib = L.lib()
    b = interior_random(3, 25, 21)
    ref = tps.PoissonProblem(3, 3, 8)
    x_ref, r_ref = tps.MultigridSolvers(ref).solve_cg(b, precision="fp32", rel_tol=1e-10)
    ref.close()
    P = tps.PoissonProblem(3, 3, 8)
    failures = 0
    try:
        for n in range(1, 400):
            x = torch.zeros_like(b)
            lib.tps_inject_alloc_failure(n)
            st, rep = raw_solve(P, b, x)
            lib.tps_inject_alloc_failure(0)
            if st == L.TPS_OK:
                break
            assert st == ALLOC, (n, st)
            assert b"injected" in lib.tps_last_error(P.handle)
            failures += 1
    finally:
        lib.tps_inject_alloc_failure(0)
    assert st == L.TPS_OK and failures >= 3
    assert rep.iterations == r_ref.iterations
    assert torch.equal(x, x_ref)
    # GMRES allocates its basis lazily as well
    lib.tps_inject_alloc_failure(1)
    st, _ = raw_solve(P, b, torch.zeros_like(b), driver=L.DRIVER_GMRES, precision=L.VCYCLE_F64_ROUNDED,
                      max_iter=20, rel_tol=1e-8)
    lib.tps_inject_alloc_failure(0)
    assert st == ALLOC
    st, rep = raw_solve(P, b, torch.zeros_like(b), driver=L.DRIVER_GMRES, precision=L.VCYCLE_F64_ROUNDED,
                        max_iter=20, rel_tol=1e-8)
    assert st in (L.TPS_OK, NOT_CONVERGED) and rep.iterations >= 1
    P.close()


def test_injected_allocation_failure_in_batch_create(cuda):
    lib = L.lib()
    lib.tps_inject_alloc_failure(1)
    try:
        with pytest.raises(tps.TpsError) as ei:
            tps.BatchSolver([(3, 3, 8), (3, 2, 6)])
    finally:
        lib.tps_inject_alloc_failure(0)
    assert ei.value.status == ALLOC
    B = tps.BatchSolver([(3, 3, 8), (3, 2, 6)])
    xs, reps = B.solve([interior_random(3, 25, 1), interior_random(3, 13, 2)], precision="fp32")
    assert all(r.converged for r in reps)
    B.close()


def test_rejected_kappa_keeps_the_coefficient(cuda):
    """tps_set_kappa validates before it changes anything: a negative value is
    rejected and the solve afterwards still uses the previous coefficient."""
    n = 8
    rng = np.random.default_rng(4)
    kappa = rng.uniform(0.5, 2.0, n ** 3)
    P = tps.PoissonProblem(3, 2, n, kappa=kappa)
    b = interior_random(3, 17, 8)
    x1, r1 = tps.MultigridSolvers(P).solve_cg(b, precision="fp64", rel_tol=1e-10)
    bad = kappa.copy()
    bad[17] = -1.0
    with pytest.raises(tps.TpsError) as ei:
        P.set_kappa(bad)
    assert ei.value.status == INVALID
    x2, r2 = tps.MultigridSolvers(P).solve_cg(b, precision="fp64", rel_tol=1e-10)
    assert r2.iterations == r1.iterations and torch.equal(x1, x2)
    P.close()


def test_bounded_wait_timeout_reaches_the_host(cuda):
    lib = L.lib()
    P = tps.PoissonProblem(3, 3, 8)
    h, s = P.handle, stream()
    assert lib.tps_device_status(h) == L.TPS_OK
    # asynchronous: the launch itself succeeds, the timeout is found by the check
    assert lib.tps_selftest_wait_timeout(h, SHORT_WAIT, s) == L.TPS_OK
    assert lib.tps_device_status(h) == TIMEOUT
    assert b"bounded device wait" in lib.tps_last_error(h)
    assert lib.tps_device_status(h) == L.TPS_OK  # read and cleared
    assert lib.tps_selftest_wait_timeout(h, SHORT_WAIT, s) == L.TPS_OK
    with pytest.raises(tps.TpsError) as ei:
        P.check_device()
    assert ei.value.status == TIMEOUT
    # a solve picks up a timeout recorded by an earlier asynchronous call ...
    b = interior_random(3, 25, 31)
    x_ref, r_ref = tps.MultigridSolvers(P).solve_cg(b, precision="fp32", rel_tol=1e-10)
    assert lib.tps_selftest_wait_timeout(h, SHORT_WAIT, s) == L.TPS_OK
    x = torch.zeros_like(b)
    st, rep = raw_solve(P, b, x)
    assert st == TIMEOUT and not rep.converged
    # ... and the context and handle stay usable: the next solve is exact
    x = torch.zeros_like(b)
    st, rep = raw_solve(P, b, x)
    assert st == L.TPS_OK and rep.iterations == r_ref.iterations and torch.equal(x, x_ref)
    assert lib.tps_selftest_wait_timeout(h, SHORT_WAIT, s) == L.TPS_OK
    with pytest.raises(tps.TpsError) as ei:
        P.time_smoother(dtype="fp32", sweeps=2)
    assert ei.value.status == TIMEOUT
    assert P.time_smoother(dtype="fp32", sweeps=2) > 0.0
    # the host-buffer solve reports it too and does not copy a result back
    assert lib.tps_selftest_wait_timeout(h, SHORT_WAIT, s) == L.TPS_OK
    torch.cuda.synchronize()
    o = L.TpsSolveOpts(L.DRIVER_CG, L.VCYCLE_F32, 1, 100, 1e-10, 1e-300, 1)
    bh = b.cpu()
    xh = torch.full_like(bh, 3.0)
    r = L.TpsReport()
    assert lib.tps_solve_host_guess(h, ctypes.byref(o), bh.data_ptr(), None, xh.data_ptr(), ctypes.byref(r)) == TIMEOUT
    assert torch.all(xh == 3.0)
    P.close()


def test_bounded_wait_timeout_in_a_batch(cuda):
    lib = L.lib()
    B = tps.BatchSolver([(3, 3, 8), (3, 2, 6)])
    rhs = [interior_random(3, 25, 41), interior_random(3, 13, 42)]
    xs_ref, reps_ref = B.solve(rhs, precision="fp32")
    h1 = ctypes.c_void_p()
    assert lib.tps_batch_system(B._h, 1, ctypes.byref(h1)) == L.TPS_OK
    assert lib.tps_selftest_wait_timeout(h1, SHORT_WAIT, stream()) == L.TPS_OK
    torch.cuda.synchronize()  # the batch runs on a stream of its own
    with pytest.raises(tps.TpsError) as ei:
        B.solve(rhs, precision="fp32")
    assert ei.value.status == TIMEOUT
    xs, reps = B.solve(rhs, precision="fp32")
    for a, r, a0, r0 in zip(xs, reps, xs_ref, reps_ref):
        assert r.converged and r.iterations == r0.iterations and torch.equal(a, a0)
    B.close()
