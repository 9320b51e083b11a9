"""bench.py's multi-process plumbing on CPU (gloo, world size 2): the
rendezvous from the torchrun environment, the barrier, the max-over-ranks
timing reduction, and the reference arm's rule that only rank 0 runs and
prints.  Replicas share no data-path collective, so this is all the host
logic the multi-GPU path has."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
ws, rank, local = bench.dist_env()
dist = bench.init_dist(ws, "gloo")
bench.barrier(dist)
m = bench.max_over_ranks(dist, float(10 + rank))
print(json.dumps({{"rank": rank, "ws": ws, "max": m}}), flush=True)
dist.destroy_process_group()
"""


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def launch(code, ws=2, extra_env=None):
    port = free_port()
    procs = []
    for r in range(ws):
        env = dict(os.environ, WORLD_SIZE=str(ws), RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_max_over_ranks_and_barrier():
    outs = launch(WORKER.format(root=ROOT))
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in res) == [0, 1]
    assert all(r["ws"] == 2 and r["max"] == 11.0 for r in res)


def test_reference_arm_runs_on_rank_0_only():
    """--impl reference under a 2-rank launch: rank 1 exits 0 silently; rank
    0 prints one JSON line (a bounded sample, or the unavailable line)."""
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); sys.argv = ['bench.py', '--impl', 'reference', "
            "'--steps', '1', '--warmup', '0', '--geometry', 'small']; import bench; bench.main()")
    outs = launch(code)
    assert outs[1].strip() == ""
    line = json.loads(outs[0].strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" not in line:
        assert line["value"] > 0 and line["cpu_baseline"]["cores"] >= 1
