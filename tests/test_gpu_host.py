"""GPU tests of the host-buffer solve entry points (tps_solve_host and
tps_solve_host_guess): the copies in and out around the same MG-CG as the
device-buffer tps_solve."""
import ctypes

import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import _lib as L

pytestmark = pytest.mark.gpu


def interior_random(N1, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, N1 ** 3)
    idx = np.stack(np.unravel_index(np.arange(N1 ** 3), (N1,) * 3))
    v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return torch.tensor(v)


@pytest.mark.parametrize("precision", [L.VCYCLE_F32, L.VCYCLE_F64])
def test_host_solves_match_device_solve(cuda, precision):
    k, n = 3, 8
    P = tps.PoissonProblem(3, k, n)
    b = interior_random(n * k + 1, 11)
    x_dev, rep = tps.MultigridSolvers(P).solve_cg(b.cuda(), precision="fp32" if precision == L.VCYCLE_F32 else "fp64",
                                                  rel_tol=1e-10)
    x_dev = x_dev.cpu()
    o = L.TpsSolveOpts(L.DRIVER_CG, precision, 1, 100, 1e-10, 1e-300, 1)
    r = L.TpsReport()
    bh = b.clone().pin_memory()
    # in/out initial guess, zero
    xh = torch.zeros_like(bh).pin_memory()
    L.check(L.lib().tps_solve_host(P.handle, ctypes.byref(o), bh.data_ptr(), xh.data_ptr(), ctypes.byref(r)),
            P.handle)
    assert r.converged and r.iterations == rep.iterations
    scale = x_dev.abs().max().item()
    assert (xh - x_dev).abs().max().item() <= 1e-12 * scale
    # no guess: the solve starts from zero on the device, x_host is output only
    xo = torch.full_like(bh, 7.0).pin_memory()
    L.check(L.lib().tps_solve_host_guess(P.handle, ctypes.byref(o), bh.data_ptr(), None, xo.data_ptr(),
                                         ctypes.byref(r)), P.handle)
    assert r.converged and r.iterations == rep.iterations
    assert (xo - x_dev).abs().max().item() <= 1e-12 * scale
    # a separate guess that is already the solution: at most one iteration
    x0 = x_dev.clone().pin_memory()
    L.check(L.lib().tps_solve_host_guess(P.handle, ctypes.byref(o), bh.data_ptr(), x0.data_ptr(), xo.data_ptr(),
                                         ctypes.byref(r)), P.handle)
    assert r.converged and r.iterations <= 1
    assert torch.equal(x0, x_dev)  # the guess buffer is not written
    assert (xo - x_dev).abs().max().item() <= 1e-9 * scale
    with pytest.raises(tps.TpsError):
        L.check(L.lib().tps_solve_host_guess(P.handle, ctypes.byref(o), None, None, xo.data_ptr(),
                                             ctypes.byref(r)), P.handle)
    P.close()


def test_host_solve_sequence_matches_single_solves(cuda):
    """tps_solve_host_many: the overlapped sequence gives, for every right-hand
    side, exactly the solve of tps_solve_host_guess from zero; pinned and
    pageable buffers give the same results."""
    k, n = 3, 8
    P = tps.PoissonProblem(3, k, n)
    N1 = n * k + 1
    bs = [interior_random(N1, 20 + i) for i in range(5)]
    o = L.TpsSolveOpts(L.DRIVER_CG, L.VCYCLE_F32, 1, 100, 1e-10, 1e-300, 1)
    singles = []
    for b in bs:
        xh = torch.zeros_like(b)
        r = L.TpsReport()
        L.check(L.lib().tps_solve_host_guess(P.handle, ctypes.byref(o), b.data_ptr(), None, xh.data_ptr(),
                                             ctypes.byref(r)), P.handle)
        singles.append((xh, r.iterations))
    MG = tps.MultigridSolvers(P)
    for pinned in (True, False):
        bb = [b.clone().pin_memory() if pinned else b.clone() for b in bs]
        xs = [torch.full_like(b, 5.0) for b in bs]
        if pinned:
            xs = [x.pin_memory() for x in xs]
        xs, reps = MG.solve_host_many(bb, xs, precision="fp32", rel_tol=1e-10)
        for (x1, it1), x, r in zip(singles, xs, reps):
            assert r.converged and r.iterations == it1
            assert torch.equal(x, x1)
    # one right-hand side, default (pinned) outputs
    xs, reps = MG.solve_host_many(bs[:1])
    assert torch.equal(xs[0], singles[0][0])
    P.close()


def test_host_solve_sequence_reports_failures(cuda):
    k, n = 3, 8
    P = tps.PoissonProblem(3, k, n)
    N1 = n * k + 1
    bs = [interior_random(N1, 30 + i).pin_memory() for i in range(3)]
    bs[1][N1 * N1 * 12 + N1 * 12 + 12] = float("nan")
    xs = [torch.full_like(b, 5.0).pin_memory() for b in bs]
    o = L.TpsSolveOpts(L.DRIVER_CG, L.VCYCLE_F32, 1, 100, 1e-10, 1e-300, 1)
    reps = (L.TpsReport * 3)()
    bp = (ctypes.c_void_p * 3)(*[b.data_ptr() for b in bs])
    xp = (ctypes.c_void_p * 3)(*[x.data_ptr() for x in xs])
    st = L.lib().tps_solve_host_many(P.handle, ctypes.byref(o), 3, bp, xp, reps)
    assert st == 6  # TPS_ERR_NONFINITE
    assert reps[0].converged and reps[2].converged and not reps[1].converged
    assert torch.all(xs[1] == 5.0)  # no result copied for the failed solve
    MG = tps.MultigridSolvers(P)
    x0, _ = MG.solve_cg(bs[0].cuda(), precision="fp32", rel_tol=1e-10)
    x2, _ = MG.solve_cg(bs[2].cuda(), precision="fp32", rel_tol=1e-10)
    assert torch.equal(xs[0], x0.cpu()) and torch.equal(xs[2], x2.cpu())
    # argument errors
    assert L.lib().tps_solve_host_many(P.handle, ctypes.byref(o), 0, bp, xp, reps) == 1
    bp[1] = None
    assert L.lib().tps_solve_host_many(P.handle, ctypes.byref(o), 3, bp, xp, reps) == 1
    P.close()
