"""The N > 1 path of bench.py on the CPU: two gloo ranks (127.0.0.1) take
the max over ranks of their step times with one all-reduce and compute the
whole-job throughput of independent replicas; the reference arm's other
ranks exit without output."""
import datetime
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    got = bench.max_over_ranks(dist, [10.0 + rank, 5.0 - rank], torch.device("cpu"))
    dist.barrier()
    q.put((rank, got, bench.replica_value(world, 1000, got[0])))
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, value in out:
        assert got == [11.0, 5.0]
        assert value == pytest.approx(2 * 1000 / 11e-3)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, [3.0, 4.0], None) == [3.0, 4.0]
    assert bench.replica_value(1, 500, 2.0) == pytest.approx(250000.0)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
