"""N > 1 host logic on CPU ranks (gloo, world size 2): the replica bench's
max-over-ranks timing and the reference arm's rank-0-only rule."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["ROOT"])
import bench
class A: pass
world, rank, local, pg = bench.dist_setup(A())
v = bench.max_over_ranks(pg, float(rank + 1) * 1.5)
bench.barrier(pg)
print(json.dumps({"rank": rank, "world": world, "max": v}), flush=True)
pg.destroy_process_group()
"""


def run_ranks(code, world=2, extra_env=None):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, ROOT=ROOT, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_max_over_ranks_gloo():
    outs = run_ranks(WORKER)
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert all(r["world"] == 2 and r["max"] == 3.0 for r in res)


def test_reference_arm_rank0_only():
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                                       "--gpus", "2", "--steps", "1", "--warmup", "0", "--n", "32",
                                       "--ref-seconds", "0.3"], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=300)
        assert p.returncode == 0, e
        outs.append(o.strip())
    line = json.loads(outs[0].splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
    assert outs[1] == ""
