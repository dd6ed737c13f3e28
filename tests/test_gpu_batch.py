"""GPU tests of the batched solver (tps_batch_*): many right-hand sides and
meshes of different sizes in one graph launch must give exactly the solves
of the single-system driver (same iteration counts, same solutions)."""
import numpy as np
import pytest
import torch

import gputensorproductsmoother_b200 as tps

pytestmark = pytest.mark.gpu


def interior_random(dim, N1, seed):
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1, 1, N1 ** dim)
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    v[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0.0
    return torch.tensor(v, device="cuda")


SYSTEMS = [(3, 3, 8)] * 3 + [(3, 3, 6), (3, 3, 12), (3, 2, 10), (2, 3, 16), (3, 4, 4)]


@pytest.mark.parametrize("precision", ["fp64", "fp32", "tf32"])
def test_batch_matches_single_solves(cuda, precision):
    systems = SYSTEMS if precision != "tf32" else [s for s in SYSTEMS if s[0] == 3]
    B = tps.BatchSolver(systems)
    rhs = [interior_random(d, n * k + 1, 10 + i) for i, (d, k, n) in enumerate(systems)]
    xs, reps = B.solve(rhs, precision=precision, rel_tol=1e-10)
    for i, (d, k, n) in enumerate(systems):
        P = tps.PoissonProblem(d, k, n)
        x1, r1 = tps.MultigridSolvers(P).solve_cg(rhs[i], precision=precision, rel_tol=1e-10)
        assert reps[i].converged and reps[i].final_residual <= 1e-10
        assert reps[i].iterations == r1.iterations, (i, reps[i].iterations, r1.iterations)
        np.testing.assert_allclose(reps[i].history, r1.history, rtol=1e-9, atol=0)
        e = (xs[i] - x1).abs().max().item() / x1.abs().max().item()
        assert e < 1e-12, (i, e)
        P.close()
    # a second launch reuses the instantiated graph and gives the same result
    xs2, reps2 = B.solve(rhs, x=[torch.zeros_like(b) for b in rhs], precision=precision, rel_tol=1e-10)
    for i in range(len(systems)):
        assert reps2[i].iterations == reps[i].iterations
        assert torch.equal(xs2[i], xs[i]) or (xs2[i] - xs[i]).abs().max().item() == 0.0
    B.close()


def test_batch_max_iter_and_zero_rhs(cuda):
    systems = [(3, 3, 8), (3, 3, 8)]
    B = tps.BatchSolver(systems)
    rhs = [interior_random(3, 25, 1), torch.zeros(25 ** 3, dtype=torch.float64, device="cuda")]
    xs, reps = B.solve(rhs, precision="fp32", rel_tol=1e-14, max_iter=2, raise_on_fail=False)
    assert reps[0].iterations == 2 and not reps[0].converged
    # b = 0: converged at iteration 0 with x = 0, never enters the loop body
    assert reps[1].iterations == 0 and reps[1].converged
    assert xs[1].abs().max().item() == 0.0
    with pytest.raises(tps.TpsError):
        B.solve(rhs, precision="fp32", rel_tol=1e-14, max_iter=2)
    B.close()


def test_autotune_keeps_results(cuda):
    """The kernel variants only regroup independent patches of a colour: the
    autotuned sweep is bit-identical to the default one."""
    P = tps.PoissonProblem(3, 3, 16)
    N1 = 49
    x0, b = interior_random(3, N1, 1).float(), interior_random(3, N1, 2).float()
    x_def = x0.clone()
    tps.PatchSmoother(P).step(x_def, b)
    ppb = P.autotune("fp32")
    assert len(ppb) == P.n_levels and all(v >= 1 or v in (-1, -2) for v in ppb)
    x_tuned = x0.clone()
    tps.PatchSmoother(P).step(x_tuned, b)
    torch.cuda.synchronize()
    assert torch.equal(x_tuned, x_def)
    MG = tps.MultigridSolvers(P)
    bb = interior_random(3, N1, 3)
    x, rep = MG.solve_cg(bb, precision="fp32", rel_tol=1e-10)
    assert rep.converged
    assert P.autotune("fp64")[0] in (-1, 1, 2, 4, 8, 16)


def test_autotune_operator_tile_depth_keeps_results(cuda):
    """The autotuner also picks the operator's cell layers per CTA (1, 2, 4, 8
    or 16, at most the level's cells).  Every output of the operator is formed by
    the same arithmetic whatever the tile depth, so the mat-vec is
    bit-identical; the CG's fused p.q is summed per CTA, so its rounding
    follows the tile depth: solves after tuning take the same iterations and
    agree to rounding (each configuration is itself deterministic)."""
    P = tps.PoissonProblem(3, 4, 16)
    N1 = 65
    bb = interior_random(3, N1, 4)
    MG = tps.MultigridSolvers(P)
    A = tps.LaplaceOperator(P)
    src = interior_random(3, N1, 5)
    y_ref = torch.empty_like(src)
    A.vmult(y_ref, src)
    ref = {p: MG.solve_cg(bb, precision=p, rel_tol=1e-10) for p in ("fp32", "fp64")}
    assert all(P.operator_layers(lv, dt) == 0 for lv in range(P.n_levels) for dt in ("fp32", "fp64"))
    P.autotune("fp32")
    P.autotune("fp64")
    for dt in ("fp32", "fp64"):
        for lv in range(P.n_levels):
            cz = P.operator_layers(lv, dt)
            assert cz in (1, 2, 4, 8, 16) and cz <= P.cells(lv), (dt, lv, cz)
    for cz in (1, 2, 4, 8, 16):  # every tile depth of the finest level: the same mat-vec
        P.set_operator_layers(cz, "fp64", P.n_levels - 1)
        y = torch.empty_like(src)
        A.vmult(y, src)
        assert torch.equal(y, y_ref), cz
    with pytest.raises(tps.TpsError):
        P.set_operator_layers(3, "fp64", 0)
    P.autotune("fp64")
    for p in ("fp32", "fp64"):
        x, rep = MG.solve_cg(bb, precision=p, rel_tol=1e-10)
        assert rep.iterations == ref[p][1].iterations
        d = ((x - ref[p][0]).norm() / ref[p][0].norm()).item()
        assert d <= 1e-12, (p, d)
        x2, _ = MG.solve_cg(bb, precision=p, rel_tol=1e-10)
        assert torch.equal(x2, x), p
