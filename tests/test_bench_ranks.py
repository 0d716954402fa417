"""The bench's multi-rank plumbing on CPU: two gloo ranks (one process per GPU
on a B200 node) combine their timed seconds by max and their counted ground
states by sum; the reference arm runs on rank 0 only. Also the bench's byte
accounting for the roofline (complex64 fields in the mixed form's FP32 phase)."""
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


def _part(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        insts = bench._instances("c4")
        ref = bench._reference_runs()
        mine = bench.partition(insts, ref, 2, rank)
        # each rank solves its share alone; the counts meet only in job_rate
        out[rank] = (mine, bench.job_rate(1.0 + rank, len(mine), dist, "cpu"))
    finally:
        dist.destroy_process_group()


def test_partition_over_two_gloo_ranks_covers_the_workload_once():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_part, args=(port, out), nprocs=2, start_method="spawn", join=True)
        res = dict(out)
    a, b = res[0][0], res[1][0]
    assert sorted(a + b) == list(range(64)) and not set(a) & set(b)
    insts, ref = bench._instances("c4"), bench._reference_runs()
    # the four long instances (reference iterations > 10000) are split evenly
    tail = [i for i, p in enumerate(insts) if ref[p["name"]]["obs"]["iters"] > 10000]
    assert len(set(tail) & set(a)) == 2 and len(set(tail) & set(b)) == 2
    assert res[0][1] == res[1][1] == (2.0, 64.0, 32.0)


def test_reference_rotation_covers_every_instance_once():
    insts, ref = bench._instances("c4"), bench._reference_runs()
    for steps, procs in ((20, 16), (3, 8), (1, 4), (100, 8)):
        g = bench.rotation_groups(insts, ref, steps, procs)
        names = [p["name"] for grp in g for p in grp]
        assert sorted(names) == sorted(p["name"] for p in insts)
        assert len(g) <= steps
        # the costliest instances run side by side in the first step
        top = sorted(insts, key=lambda p: -bench._cost(p, ref))[:procs]
        assert [p["name"] for p in g[0][:procs]] == [p["name"] for p in top]


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


def test_algorithmic_bytes_follow_the_storage_precision():
    import bench
    full = bench.algorithmic_bytes(2, 256 * 256, 100, 80, 130)
    # FP64 throughout: 16-byte fields
    assert bench.algorithmic_bytes(2, 256 * 256, 100, 80, 130, 0) == full
    # complex64 throughout: the field bytes halve, the 8-byte keys and potential do not
    half = bench.algorithmic_bytes(2, 256 * 256, 100, 80, 130, 100)
    assert 0.5 * full < half < 0.55 * full
    # a hand-over half way lies in between, linearly
    mid = bench.algorithmic_bytes(2, 256 * 256, 100, 80, 130, 50)
    assert abs(mid - 0.5 * (full + half)) <= 1e-9 * full

    class R:
        iters, fp64_from = 40, -1
    assert bench.fp32_iterations(R) == 40
    R.fp64_from = 0
    assert bench.fp32_iterations(R) == 0
    R.fp64_from = 17
    assert bench.fp32_iterations(R) == 17
