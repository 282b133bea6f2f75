"""Multi-rank plumbing of bench.py on the CPU (gloo, world size 2).

The path runs as replicas (one independent imageFiltering task per GPU, no
data-path collective): what ranks share is the barrier around the timed
region, the max of the per-rank device times, and the whole-job rate.  The
same `bench.Ranks` code runs over NCCL on the GPU box; here two processes
rendezvous on 127.0.0.1 over gloo.  The reference arm runs on rank 0 only.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
import types

from conftest import ROOT

WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
r = bench.Ranks("gloo")
slowest = r.max(10.0 + r.rank)            # rank 1 is the slow one
r.barrier()
rate = r.rate(1e9, 2, 2000.0)             # 1e9 units per rank per step, 2 steps, 2 s
world, rank = r.world, r.rank
r.close()
print(json.dumps({"rank": rank, "world": world, "max": slowest, "rate": rate}))
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_max_and_rate():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(o["rank"] for o in outs) == [0, 1]
    for o in outs:
        assert o["world"] == 2
        assert o["max"] == 11.0
        assert abs(o["rate"] - 2.0) < 1e-12      # 2 ranks x 1 G units/s


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, ROOT)
    import bench

    r = bench.Ranks("gloo")
    assert r.world == 1 and r.dist is None
    assert r.max(3.5) == 3.5
    assert abs(r.rate(402653184, 20, 100.0) - 80.5306368) < 1e-9
    r.barrier()
    r.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    sys.path.insert(0, ROOT)
    import bench

    args = types.SimpleNamespace(gpus=2, steps=1, warmup=3)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""
