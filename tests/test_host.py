"""CPU tests of the host-side helpers: mesh hierarchy splitting, the seeded
workload generators and the benchmark's algorithmic-byte model."""
import numpy as np
import pytest
import torch

import bench
from gputensorproductsmoother_b200 import problems, split_cells


@pytest.mark.parametrize("n,expect", [(2, (2, 1)), (64, (2, 6)), (48, (3, 5)), (32, (2, 5)),
                                      (12, (3, 3)), (5, (5, 1))])
def test_split_cells(n, expect):
    assert split_cells(n) == expect


def test_split_cells_rejects_one_cell():
    with pytest.raises(ValueError):
        split_cells(1)


def test_gauss_lobatto_nodes_match_oracle(oracle):
    for k in range(1, 8):
        assert np.allclose(problems.gauss_lobatto(k), oracle.fe1d(k)[0], atol=1e-14)


def test_sine_rhs_matches_direct_quadrature():
    dim, k, n = 3, 2, 4
    b = problems.sine_modes_rhs(dim, k, n, seed=3, device="cpu").numpy()
    rng = np.random.default_rng(3)
    amps = rng.uniform(-1, 1, 8)
    freqs = rng.integers(1, 9, size=(8, dim))
    N1 = n * k + 1
    ref = np.zeros((N1,) * dim)
    for a, f in zip(amps, freqs):
        v = [problems.load_1d_sin(k, n, int(fi)) for fi in f]
        ref += a * np.einsum("z,y,x->zyx", v[2], v[1], v[0])
    ref = ref.ravel()
    idx = np.stack(np.unravel_index(np.arange(N1 ** dim), (N1,) * dim))
    ref[np.any((idx == 0) | (idx == N1 - 1), axis=0)] = 0
    assert np.allclose(b, ref, atol=1e-14)


def test_nodal_rhs_is_mass_times_f():
    dim, k, n = 2, 2, 4
    b = problems.nodal_rhs(dim, k, n, seed=1, device="cpu").numpy()
    M = problems.mass_1d(k, n)
    N1 = n * k + 1
    f = np.random.default_rng(1).uniform(-1, 1, N1 ** 2).reshape(N1, N1)
    f[0, :] = f[-1, :] = f[:, 0] = f[:, -1] = 0
    ref = M @ f @ M.T
    ref[0, :] = ref[-1, :] = ref[:, 0] = ref[:, -1] = 0
    assert np.allclose(b.reshape(N1, N1), ref, atol=1e-15)


@pytest.mark.parametrize("dim,k,n", [(2, 2, 4), (3, 2, 6), (3, 4, 5)])
def test_smoother_byte_model_counts_unions(dim, k, n):
    """s(|U_c| + 2|I_c|) equals an explicit union count over the colour's patches."""
    total, per = bench.smoother_bytes(dim, k, n, 1)
    N1 = n * k + 1
    for c in range(1 << dim):
        box = np.zeros((N1,) * dim, bool)
        inter = np.zeros((N1,) * dim, bool)
        par = [(c >> d) & 1 for d in range(dim)]
        for p in np.ndindex(*([n - 1] * dim)):
            if any((p[d] & 1) != par[d] for d in range(dim)):
                continue
            sl = tuple(slice(p[d] * k, p[d] * k + 2 * k + 1) for d in range(dim))[::-1]
            si = tuple(slice(p[d] * k + 1, p[d] * k + 2 * k) for d in range(dim))[::-1]
            box[sl] = True
            inter[si] = True
        assert per[c] == box.sum() + 2 * inter.sum()


def test_launch_model_is_positive():
    assert bench.launches_per_solve(3, 6, 6) > bench.launches_per_solve(3, 6, 1) > 0


@pytest.mark.parametrize("dim", [2, 3])
def test_colouring_is_race_free(dim):
    """Host bitmap check of the 2^d colouring (tps_check_colouring): every
    interior vertex is one patch centre, same-colour interiors are disjoint
    and no box ring read by a colour meets an interior it writes, for every
    degree and odd, even and non-power-of-two meshes."""
    from gputensorproductsmoother_b200 import _lib as L
    lib = L.lib()
    for k in range(1, 8):
        for n in (2, 3, 4, 5, 6, 8, 12, 16) if dim == 3 else (2, 3, 4, 5, 7, 8, 16, 24, 64):
            assert lib.tps_check_colouring(dim, k, n) == 0, (dim, k, n, lib.tps_last_error(None))


def test_colouring_check_rejects_bad_arguments():
    from gputensorproductsmoother_b200 import _lib as L
    lib = L.lib()
    assert lib.tps_check_colouring(4, 2, 8) == 1
    assert lib.tps_check_colouring(3, 0, 8) == 1
    assert lib.tps_check_colouring(3, 2, 1) == 1
    assert b"tps_check_colouring" in lib.tps_last_error(None)


def test_bench_config_file(tmp_path, monkeypatch):
    """bench.py --config: JSON option values, command-line options win,
    unknown keys are rejected."""
    import json
    import sys
    cfg = tmp_path / "c.json"
    cfg.write_text(json.dumps({"mode": "smoother", "steps": 2, "no-cpu-baseline": True}))
    monkeypatch.setattr(sys, "argv", ["bench.py", "--config", str(cfg), "--steps", "5"])
    a = bench.parse()
    assert (a.mode, a.steps, a.no_cpu_baseline, a.warmup) == ("smoother", 5, True, 3)
    cfg.write_text(json.dumps({"stepz": 2}))
    monkeypatch.setattr(sys, "argv", ["bench.py", "--config", str(cfg)])
    with pytest.raises(SystemExit):
        bench.parse()
