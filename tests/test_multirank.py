"""N > 1 host logic on CPU ranks (gloo, world size 2 and 3): the bench's
max-over-ranks timing, the reference arm's rank-0-only rule, and the rank
contexts' exchange protocol -- each rank plans its own context (the
library's host-only dry run of octlb_gpu_create_part) and the lists it would
send travel over gloo to the peers, which check them against the lists they
expect to receive, in order."""
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


EXCH = r"""
import os, sys, json
sys.path.insert(0, os.environ["ROOT"])
import numpy as np
import torch
import torch.distributed as dist
from datetime import timedelta
dist.init_process_group("gloo", timeout=timedelta(seconds=60))
rank, world = dist.get_rank(), dist.get_world_size()
import octlb_b200 as ob
from octlb_b200 import cases
mesh, init, info = (cases.cylinder_forest() if os.environ["CASE"] == "cylinder"
                    else cases.cavity_forest(cells=64, n=8, lid=0.05, tau=0.56, band_cells=8))
owner = ob.partition(mesh, world)
links = os.environ["CASE"] == "cylinder"
recs = ob.plan_part(mesh, info["omega"], rank, owner, stream_mode=ob.STREAM_LINKS if links else ob.STREAM_ROTATE,
                    drag=links)
checked = 0
for kind_send, kind_recv in ((0, 1), (2, 3)):
    for src in range(world):
        for dst in range(world):
            if src == dst:
                continue
            if rank == src:
                mine = recs[(recs[:, 1] == kind_send) & (recs[:, 2] == dst)][:, [0, 3]]
                n = torch.tensor([len(mine)], dtype=torch.int64)
                dist.send(n, dst)
                if len(mine):
                    dist.send(torch.from_numpy(np.ascontiguousarray(mine)), dst)
            elif rank == dst:
                n = torch.zeros(1, dtype=torch.int64)
                dist.recv(n, src)
                got = torch.zeros((int(n), 2), dtype=torch.int64)
                if int(n):
                    dist.recv(got, src)
                want = recs[(recs[:, 1] == kind_recv) & (recs[:, 2] == src)][:, [0, 3]]
                assert np.array_equal(got.numpy(), want), (src, dst, kind_send, len(got), len(want))
                checked += len(want)
            dist.barrier()
print(json.dumps({"rank": rank, "checked": checked, "records": int(len(recs))}), flush=True)
dist.destroy_process_group()
"""


@pytest.mark.parametrize("case,world", [("cylinder", 2), ("amr", 3)])
def test_rank_exchange_lists_agree_over_gloo(case, world):
    outs = run_ranks(EXCH, world=world, extra_env={"CASE": case})
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert all(r["checked"] > 0 for r in res)
