"""bench.py's multi-rank logic on the CPU: two gloo ranks (127.0.0.1) shard the BFS source
order so that every source lands on exactly one rank, and a timing is the max over ranks on
every rank. (On the GPUs the same functions run over NCCL with one process per GPU.)"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np

import bench


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, order, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        share = bench.shard_sources(order, world, rank)
        shares = [None] * world
        dist.all_gather_object(shares, share.tolist())
        slowest = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
        dist.barrier()
        q.put((rank, shares, slowest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_every_source_once_and_time_the_slowest():
    world = 2
    order = np.random.default_rng(0).permutation(1001)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, order, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, shares, slowest in got:
        assert slowest == 10.0 * world
        assert np.array_equal(np.concatenate([np.asarray(s) for s in shares]), order)
        assert abs(len(shares[0]) - len(shares[1])) <= 1
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_launch_ranks_starts_one_process_per_rank(capfd):
    """bench.launch_ranks (what `bench.py --gpus N` uses when no launcher started it) runs N ranks
    under torch.distributed.run on 127.0.0.1; here two gloo ranks of a probe script."""
    probe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rank_probe.py")
    rc = bench.launch_ranks(probe, ["1001"], 2, timeout_s=240)
    assert rc == 0
    lines = [ln for ln in capfd.readouterr().out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    import json

    got = json.loads(lines[0])
    assert got["n_gpus"] == 2 and got["parallelism"] == "replicas2"
    assert sum(got["ranks_sources"]) == 1001 and got["slowest"] == 2.0


def test_bench_refuses_a_world_size_that_is_not_gpus(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "3")
    assert bench.main(["--gpus", "2", "--steps", "1"]) == 2
