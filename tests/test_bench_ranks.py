"""The bench's multi-rank plumbing on CPU: two gloo ranks (one process per GPU
on a B200 node) combine their timed seconds by max and their counted ground
states by sum; the reference arm runs on rank 0 only."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        total = [1.5, 2.0][rank]
        counted = [10, 7][rank]
        out[rank] = bench.job_rate(total, counted, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_job_rate_over_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(port, out), nprocs=2, start_method="spawn", join=True)
        res = dict(out)
    for r in (0, 1):
        tmax, counted, value = res[r]
        assert tmax == 2.0 and counted == 17.0 and abs(value - 8.5) < 1e-15


def test_job_rate_single_rank():
    assert bench.job_rate(2.0, 5) == (2.0, 5.0, 2.5)


def test_reference_arm_runs_on_rank0_only(capsys, monkeypatch):
    monkeypatch.setenv("RANK", "1")

    class A:
        workload = "c4"
        steps = 1
        warmup = 0
        cpu_sample = 1
        gpus = 2
    bench.run_reference(A())
    assert capsys.readouterr().out == ""
