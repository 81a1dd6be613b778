"""The N > 1 paths on the CPU, as gloo ranks on 127.0.0.1:
  * bench.py: two ranks take the max over ranks of their step times with one
    all-reduce and compute the whole-job throughput of independent replicas;
    the reference arm's other ranks exit without output;
  * the sharded fixpoint (gsc_shard.ShardedFixpoint over TorchComm): two and
    three ranks own contiguous slice ranges, exchange their slabs and summed
    counts every iteration, apply the stop rules alike and gather the result,
    which must equal the oracle's whole solve bit for bit.  The per-rank
    compute is the oracle's per-state step (tests/shard_oracle_engine.py), so
    these tests cover the partition, the exchange, the stop rules and the
    gather; the device engine runs the same loop in tests/test_gpu_shard.py."""
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


def _shard_rank(rank, world, port, name, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    for p in (os.path.join(ROOT, "gpu-inner-outer_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import gsc_shard
    from helpers import golden_index
    from shard_oracle_engine import OracleShardEngine

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        case = golden_index()[name]["case"]
        res = gsc_shard.ShardedFixpoint(OracleShardEngine(case), gsc_shard.TorchComm(dist)).run()
        q.put((rank, {k: res[k] for k in ("valid_mask", "candidate_mask", "reachable_mask", "controller",
                                           "reach_step", "iterations", "message", "iter_new_reachable",
                                           "iter_new_certified")}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("small", 2), ("hyperbolic_mid_a", 2), ("hyperbolic_mid_a", 3),
                                        ("wraparound", 2), ("default_empty_candidate", 2), ("small_maxiter0", 2)])
def test_sharded_fixpoint_over_gloo_ranks_matches_the_oracle(name, world):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import assert_same_result, golden_arrays, golden_index

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = dict(golden_arrays(name))
    meta = golden_index()[name]
    for rank in range(world):
        got = out[rank]
        assert_same_result(got, {k: want[k] for k in ("valid_mask", "candidate_mask", "reachable_mask",
                                                      "controller", "reach_step")}, f"{name} rank {rank}")
        assert got["iterations"] == meta["iterations"] and got["message"] == meta["message"]


def test_partition_covers_every_slice_once():
    sys.path.insert(0, os.path.join(ROOT, "gpu-inner-outer_b200"))
    import gsc_shard

    for slices, world in ((950, 8), (7, 3), (4, 4), (1000, 7)):
        parts = gsc_shard.partition(slices, world)
        assert parts[0][0] == 0 and parts[-1][1] == slices
        assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
        sizes = [hi - lo for lo, hi in parts]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        gsc_shard.partition(3, 4)
