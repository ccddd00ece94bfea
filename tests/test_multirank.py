"""The multi-GPU plumbing on CPU: two gloo ranks.

One impact does not partition at this size, so `bench.py --gpus N` runs N
independent replicas and the job's time is the slowest rank's (max over ranks).
These tests run that plumbing with the gloo backend on the CPU: the max-over-
ranks reduction, and the reference arm under torchrun, where rank 0 alone
times the CPU oracle and prints one line while the other ranks exit cleanly.
"""
import json
import os
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as td
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    out[rank] = bench.max_over_ranks(1.5 + rank)
    td.barrier()
    td.destroy_process_group()


def test_max_over_ranks_with_gloo():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_under_torchrun():
    port = 30500 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--particles", "16384", "--cpu-seconds", "0.5", "--steps", "4",
           "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0


def _rank_sum(rank, world, port, out):
    import datetime
    import torch.distributed as td
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    share = bench.ensemble_share(64, rank, world)
    out[rank] = (bench.sum_over_ranks(len(share)), bench.max_over_ranks(float(len(share))), share)
    td.barrier()
    td.destroy_process_group()


def test_ensemble_shards_by_instance_with_gloo():
    """The ensemble under torchrun: every impact on exactly one rank, each rank a mix of sizes, and only the
    totals reduced across ranks at the end (the summed count and the slowest rank)."""
    from cosmic_collisions_b200 import configs
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = 29700 + os.getpid() % 1000
    world = 3
    procs = [ctx.Process(target=_rank_sum, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    shares = [out[r][2] for r in range(world)]
    assert sorted(i for s in shares for i in s) == list(range(64))
    assert all(out[r][0] == 64 and out[r][1] == 22.0 for r in range(world))
    sizes = [o["N"] for o in configs.ensemble_opts(64)]
    for s in shares:
        assert len({sizes[i] for i in s}) >= 3
