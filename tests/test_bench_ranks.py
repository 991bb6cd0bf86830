"""The multi-rank path of bench.py on CPU (gloo, world size 2): each rank
advances its own shard of garments with no collective on the data path, the
job time is the maximum over ranks, and the job value counts every rank's
instances. Under --impl reference only rank 0 works and prints."""
import datetime
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = 10.0 + 5.0 * rank  # the slower rank sets the job time
    total = bench.max_over_ranks(local_ms, world, "cpu")
    specs = bench.workload(16, rank)
    q.put((rank, total, bench.job_value(len(specs), world, 4, total), [round(s.stretch, 6) for s in specs]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_the_garments_and_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, t0, v0, s0), (_, t1, v1, s1) = res
    assert t0 == t1 == 15.0
    assert v0 == v1 == 16 * 2 * 4 / 0.015
    assert s0 != s1  # each rank simulates its own garments


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
