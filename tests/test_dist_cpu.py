"""The N-GPU bench path on CPU: two gloo ranks (127.0.0.1).  Replicas only --
each rank solves its own seeded instance, nothing crosses ranks on the data
path; the timings are reduced with a maximum over ranks and the job's
throughput is the sum of the ranks' units over the slowest rank's time."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import bench
    from gputensorproductsmoother_b200 import problems
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r reports timings (r+1)*[1, 2, 3]: every rank sees the maximum
        got = bench.max_over_ranks([(rank + 1) * 1.0, (rank + 1) * 2.0, (rank + 1) * 3.0], world, "cpu")
        # replica inputs: one seed per rank, different right-hand sides
        b = problems.make_rhs("poisson2d_q2_64", seed=rank, device="cpu")
        norms = torch.zeros(world, dtype=torch.float64)
        norms[rank] = float(b.norm())
        dist.all_reduce(norms)
        out[rank] = (got, norms.tolist())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_timing_and_replica_seeds():
    world = 2
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        got, norms = out[r]
        assert got == [2.0, 4.0, 6.0]
        assert norms[0] != norms[1]  # independent seeded instances per rank


def test_job_throughput_is_total_units_over_slowest_rank():
    import bench
    assert bench.job_throughput(4, 1.0e6, 2.0) == pytest.approx(2.0e9)
    assert bench.max_over_ranks([1.0, 2.0], 1, "cpu") == [1.0, 2.0]


def test_reference_arm_non_zero_rank_does_no_work(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")
    ns = type("A", (), {"workload": "poisson2d_q2_64", "steps": 1, "warmup": 0, "gpus": 2})()
    bench.run_reference(ns)
    assert capsys.readouterr().out == ""
