"""CPU: the multi-GPU mode of bench.py is replicas: every rank reconstructs
its own batch and nothing crosses ranks on the data path; only the step
times meet, as their maximum. That host logic runs here as two gloo ranks
on 127.0.0.1: the max-over-ranks time (the same on every rank), whole-job
throughput, distinct records per rank, and the reference arm's rank-0-only
output."""
import argparse
import datetime
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, q):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        q.put((rank, bench.max_over_ranks(times[rank], dist, torch.device("cpu"))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run_ranks(times):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, len(times), port, times, q)) for r in range(len(times))]
    for p in procs:
        p.start()
    try:
        got = dict(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    return got


def test_step_time_is_the_slowest_rank_on_every_rank():
    got = _run_ranks([9.5, 12.25])
    assert got == {0: 12.25, 1: 12.25}


def test_single_process_time_is_unchanged():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(7.0, None, "cpu") == 7.0


def test_job_throughput_counts_every_replica():
    sys.path.insert(0, ROOT)
    import bench

    px = 128 * 1920 * 1080
    one = bench.job_mpx_per_s(1, px, 10.0)
    assert one == pytest.approx(px / 10e-3 / 1e6)
    assert bench.job_mpx_per_s(2, px, 10.0) == pytest.approx(2 * one)


def test_replicas_decode_different_records(pkg):
    """Each rank encodes its own content stream (same generator, different
    seed), so the replicas' batches differ."""
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    from rustmpeg_next_b200 import synth

    _, _, p = synth.workload_picture(0, 1, (27,), width=128, height=64)
    a = synth.workload_sources(0, p, stream=0)
    b = synth.workload_sources(0, p, stream=1)
    assert a[0].shape == (64, 128) and not np.array_equal(a[0], b[0])
    assert bench.rank_seed(0) != bench.rank_seed(1)


def test_reference_arm_prints_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    args = argparse.Namespace(gpus=2, steps=1, warmup=0, frames_per_qp=32)
    assert bench.run_reference(args, rank=1) is None
    assert capsys.readouterr().out == ""
