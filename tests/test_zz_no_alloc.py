"""GPU test of tps_restrict_add_noalloc, the restriction entry point for
callers that must not allocate device memory (their framework owns it all):
its output must equal the handle-based tps_restrict_add on the same inputs,
on two calls in a row (the second call reuses the library's fixed scratch
array that the first one filled).  Collected last (file name) so that a run
stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps
from gputensorproductsmoother_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,k,n_fine", [(3, 4, 8), (3, 2, 16), (2, 3, 16)])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_noalloc_restriction_matches_handle_api(cuda, dim, k, n_fine, dtype, tol):
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
        err = (out - ref).abs().max().item() / ref.abs().max().item()
        assert err <= tol, (call, err)


def test_noalloc_rejects_oversized_problem(cuda):
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = L.lib().tps_restrict_add_noalloc(3, 4, 64, L.TPS_F64, x.data_ptr(), x.data_ptr(), None)
    assert st == 1  # TPS_ERR_INVALID
    assert b"scratch" in L.lib().tps_last_error(None)
