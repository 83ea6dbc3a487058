"""bench.py with N > 1 replicas, on the CPU: the rank plumbing that torchrun
drives on N GPUs (process group, barriers, the slowest rank's figure, rank 0
alone printing; the reference arm on rank 0 only), with gloo and two ranks.
The factorization itself needs a GPU and is covered by the gpu tests."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def _free_port() -> int:
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import bench
    dist = bench.replica_group(world, backend="gloo")
    try:
        # per-rank step times: every rank gets the slowest
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        dist.barrier()
        second = bench.max_over_ranks(3.0 - rank, dist, "cpu")
        out.put((rank, slowest, second))
    finally:
        dist.destroy_process_group()


def test_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(out.get(timeout=5) for _ in range(2))
    assert got == [(0, 15.0, 3.0), (1, 15.0, 3.0)]


def test_single_process_needs_no_group():
    import bench
    assert bench.replica_group(1) is None
    assert bench.max_over_ranks(7.5, None, "cpu") == 7.5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")

    class Args:  # never read: the rank check comes first
        pass

    assert bench.run_reference(Args()) is None
    assert capsys.readouterr().out == ""
