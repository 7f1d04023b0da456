"""The multi-GPU form of bench.py is replicas: every rank solves its own batch
and rank 0 reports the whole-job rate from the slowest rank's time.  These
tests run its process-group plumbing as two gloo ranks on the CPU: the max over
ranks, the barrier, and the reference arm under torchrun (rank 0 alone prints).
"""
import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _worker(rank, ws, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    bench = _bench()
    w, r, _ = bench.dist_init()
    m = bench.all_max(1.5 * (rank + 1), w)
    bench.barrier(w)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as fh:
        json.dump({"ws": w, "rank": r, "max": m}, fh)
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for rank in range(2):
        got = json.load(open(tmp_path / f"rank{rank}.json"))
        assert got == {"ws": 2, "rank": rank, "max": 3.0}


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-threads", "2"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0 and out["cpu_baseline"]["kind"] == "port"
