"""GPU determinism tests: the kernels use no floating-point atomics (gathers,
fixed-grid two-stage reductions, disjoint same-colour patch writes), so every
operation run twice on the same inputs gives bit-identical results."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps

pytestmark = pytest.mark.gpu


def interior_random(dim, N1, seed, dtype=torch.float64):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, N1 ** dim)
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return torch.tensor(v, dtype=dtype, device="cuda")


@pytest.mark.parametrize("dim,k,n", [(2, 3, 32), (3, 4, 16), (3, 2, 32)])
@pytest.mark.parametrize("tc", [False, True])
def test_sweeps_and_solves_are_bitwise_repeatable(cuda, dim, k, n, tc):
    if tc and dim == 2:
        pytest.skip("tensor-core sweeps are 3D")
    P = tps.PoissonProblem(dim, k, n)
    N1 = n * k + 1
    x0 = interior_random(dim, N1, 1, torch.float32)
    b = interior_random(dim, N1, 2, torch.float32)
    S = tps.PatchSmoother(P, tensor_cores=tc)
    outs = []
    for _ in range(2):
        x = x0.clone()
        S.step(x, b)
        torch.cuda.synchronize()
        outs.append(x)
    assert torch.equal(outs[0], outs[1])
    MG = tps.MultigridSolvers(P)
    b64 = interior_random(dim, N1, 3)
    prec = "tf32" if tc else "fp32"
    sols = [MG.solve_cg(b64, precision=prec, rel_tol=1e-10) for _ in range(2)]
    assert sols[0][1].iterations == sols[1][1].iterations
    assert torch.equal(sols[0][0], sols[1][0])
    assert list(sols[0][1].history[:sols[0][1].iterations + 1]) == list(sols[1][1].history[:sols[1][1].iterations + 1])
    P.close()
