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
