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
