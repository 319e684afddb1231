"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1) run the max-over-ranks
timing reduction and the whole-job value exactly as the GPU ranks do with NCCL, and the
reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import datetime, json, os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
import bench
rank, world, _ = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
m = bench.max_over_ranks(ms, dist, "cpu")
v = bench.job_value(world, 1000, 8, m)
dist.barrier()
dist.destroy_process_group()
print(json.dumps({{"rank": rank, "max_ms": m, "value": v}}))
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _launch(code, world, extra_env=None, timeout=120):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True, cwd=ROOT))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=timeout)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_gloo_two_ranks_max_and_value():
    import json
    outs = _launch(RANK_SCRIPT.format(root=ROOT), 2)
    recs = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert all(r["max_ms"] == 15.0 for r in recs)
    # 2 replicas x 1000 cells x 4 stages x 8 steps in 15 ms
    assert all(abs(r["value"] - 2 * 1000 * 4 * 8 / 15e-3 / 1e9) < 1e-12 for r in recs)


def test_reference_arm_nonzero_rank_exits_without_work():
    code = ("import sys; sys.path.insert(0, %r); import bench, argparse; "
            "sys.exit(bench.run_reference(argparse.Namespace(workload='480x480x240', grid=None, steps=1, warmup=0)))"
            % ROOT)
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert r.returncode == 0 and r.stdout.strip() == ""
