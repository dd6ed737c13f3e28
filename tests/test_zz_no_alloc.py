"""GPU test of tps_restrict_add_noalloc, the restriction entry point for
callers that must not allocate device memory (their framework owns it all,
e.g. a caching allocator or an arena reserved at start-up).

* Its output must equal, bit for bit, the handle-based tps_restrict_add on
  the same inputs (both run the same kernels), on two calls in a row (the
  second call reuses the library's fixed scratch array that the first one
  filled).
* A warm call must not grow the device memory in use.
* In a fresh process, called before any handle exists (so its own first-call
  set-up runs: symbol address, context id, 1D tables), it must match the CPU
  oracle's restriction.

Collected last (file name) so that a run stopping at the first failure has
already run every other test."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import _lib as L

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("dim,k,n_fine", [(3, 4, 8), (3, 2, 16), (2, 3, 16)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_restriction_matches_handle_api(cuda, dim, k, n_fine, dtype):
    P = tps.PoissonProblem(dim, k, n_fine)
    T = tps.MGTransferCUDA(P)
    lf = P.n_levels - 1
    nc = P.cells(lf - 1)
    dt = L.TPS_F64 if dtype == torch.float64 else L.TPS_F32
    rng = np.random.default_rng(11 + dim + k)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        fine = torch.tensor(rng.uniform(-1, 1, P.n_dofs(lf)), dtype=dtype, device="cuda")
        c0 = torch.tensor(rng.uniform(-1, 1, P.n_dofs(lf - 1)), dtype=dtype, device="cuda")
        ref = c0.clone()
        T.restrict_and_add(lf, ref, fine)
        out = c0.clone()
        st = L.lib().tps_restrict_add_noalloc(dim, k, nc, dt, out.data_ptr(), fine.data_ptr(),
                                              ctypes.c_void_p(stream))
        assert st == L.TPS_OK, L.lib().tps_last_error(None)
        torch.cuda.synchronize()
        assert torch.equal(out, ref), (call, (out - ref).abs().max().item())
    P.close()


def test_noalloc_call_allocates_nothing(cuda):
    """A warm call leaves the device's free memory unchanged."""
    dim, k, nc = 3, 4, 8
    N1c, N1f = nc * k + 1, 2 * nc * k + 1
    fine = torch.rand(N1f ** 3, dtype=torch.float64, device="cuda")
    coarse = torch.zeros(N1c ** 3, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):  # warm: set-up and lazy module loading happen here
        assert L.lib().tps_restrict_add_noalloc(dim, k, nc, L.TPS_F64, coarse.data_ptr(), fine.data_ptr(),
                                                stream) == L.TPS_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert L.lib().tps_restrict_add_noalloc(dim, k, nc, L.TPS_F64, coarse.data_ptr(), fine.data_ptr(),
                                                stream) == L.TPS_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


_FRESH = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, REPO)
from gputensorproductsmoother_b200 import _lib as L
from oracle import oracle as O
rng = np.random.default_rng(5)
for dim, k, nc, dt in ((3, 3, 4, torch.float64), (2, 2, 8, torch.float32), (3, 2, 8, torch.float32)):
    N1c, N1f = nc * k + 1, 2 * nc * k + 1
    fine = rng.uniform(-1, 1, N1f ** dim)
    c0 = rng.uniform(-1, 1, N1c ** dim)
    npdt = np.float64 if dt == torch.float64 else np.float32
    ref = O.restrict_add(dim, k, nc, c0.astype(npdt), fine.astype(npdt))
    out = torch.tensor(c0, dtype=dt, device="cuda")
    fd = torch.tensor(fine, dtype=dt, device="cuda")
    code = L.TPS_F64 if dt == torch.float64 else L.TPS_F32
    st = L.lib().tps_restrict_add_noalloc(dim, k, nc, code, out.data_ptr(), fd.data_ptr(), None)
    assert st == L.TPS_OK, L.lib().tps_last_error(None)
    torch.cuda.synchronize()
    got = out.cpu().double().numpy()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    tol = 1e-12 if dt == torch.float64 else 2e-6
    assert err <= tol, (dim, k, nc, err)
print("fresh ok")
"""


def test_noalloc_first_call_in_fresh_process_matches_oracle(cuda):
    """No handle has been created in the child process: the entry point's own
    set-up runs, and its result matches the oracle's restriction (FP64 1e-12,
    FP32 2e-6 relative, the level-kernel tolerances of the parity tests)."""
    r = subprocess.run([sys.executable, "-c", "REPO = %r\n" % REPO + _FRESH], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout + r.stderr


def test_noalloc_rejects_oversized_problem(cuda):
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = L.lib().tps_restrict_add_noalloc(3, 4, 64, L.TPS_F64, x.data_ptr(), x.data_ptr(), None)
    assert st == 1  # TPS_ERR_INVALID
    assert b"scratch" in L.lib().tps_last_error(None)
    # 2D needs no scratch, but its launch grid bounds n_coarse_cells
    st = L.lib().tps_restrict_add_noalloc(2, 4, 2_000_000_000, L.TPS_F64, x.data_ptr(), x.data_ptr(), None)
    assert st == 1
    st = L.lib().tps_restrict_add_noalloc(2, 2, 600_000, L.TPS_F64, x.data_ptr(), x.data_ptr(), None)
    assert st == 1 and b"grid" in L.lib().tps_last_error(None)
