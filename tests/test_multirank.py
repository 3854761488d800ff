"""The N > 1 path of bench.py on CPU ranks (gloo, world_size 2).

The path does not need a collective on the data path: each rank renders its
own replica of the job with its own sample streams, and the only exchange is
the max over ranks of the measured times.  These tests run that reduction and
the rank-dependent pieces of the harness on two gloo processes.
"""

import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    got = bench.max_over_ranks(10.0 * (rank + 1), dist)
    seed = bench.replica_seed(rank)
    seeds = [None] * world
    dist.all_gather_object(seeds, seed)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"max": got, "seeds": seeds, "ws": bench.dist_setup()[0]}, f)


def test_max_over_ranks_and_replica_seeds(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    recs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    for r in recs:
        assert r["max"] == 20.0            # the slowest rank's time, on every rank
        assert r["ws"] == world
        assert len(set(r["seeds"])) == world   # replicas draw different sample streams


def test_reference_arm_on_other_ranks_exits_without_work():
    """Under torchrun only rank 0 times the reference; the others exit 0 silently."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0
    assert out.stdout.strip() == ""
