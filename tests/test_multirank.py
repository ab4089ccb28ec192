"""The multi-GPU layout on CPU: two gloo ranks.

The path shards by instance (independent disorder instances), so a run on N
GPUs gives each rank its own block of the global instance sequence and needs
no collective on the data path; the only collective is the max-over-ranks of
the timings. These tests run that logic as two CPU processes.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = bench.shard_instances(rank, world, 64)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # per-rank timings: the reduction must return the slowest rank's
        t = bench.max_over_ranks([10.0 + rank, 5.0 - rank], dist, "cpu")
        out[rank] = (gathered, t)
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_disjointly_and_reduce_max():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    import sys

    sys.path.insert(0, ROOT)
    import bench

    gathered, t = res[0]
    assert res[1][1] == t == [11.0, 5.0]
    seeds = [s for shard in gathered for (_, _, s) in shard]
    assert len(seeds) == len(set(seeds)) == 128
    # the union of the shards is the single-process sequence of 128 instances
    assert [i for shard in gathered for i in shard] == bench.c4_instances(128)


def test_shard_bounds():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    with pytest.raises(AssertionError):
        bench.shard_instances(2, 2, 4)
    assert bench.shard_instances(1, 4, 3) == bench.c4_instances(12)[3:6]


def test_bench_gpus_flag_launches_ranks():
    """`bench.py --gpus 2` with no torchrun environment starts its two ranks
    itself (torch.distributed.run on 127.0.0.1); the GPU leg is replaced by
    the stub leg (gloo), which keeps the sharding and the max-over-ranks
    reduction. Rank 0 prints one line for the whole job."""
    import json
    import subprocess
    import sys

    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--cpu-stub",
                        "--instances", "8"], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench

    assert d["n_gpus"] == 2 and d["instances_total"] == 16
    assert d["ms_per_step"] == 11.0  # rank 1's stand-in time: the slower rank
    assert d["seed_sum"] == float(sum(s for _, _, s in bench.c4_instances(16)))
