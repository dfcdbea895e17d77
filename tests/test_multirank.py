"""The bench's multi-rank plumbing (N independent replicas, a barrier, the
slowest rank's time) on CPU with gloo, world size 2."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys, time
sys.path.insert(0, {root!r})
import bench
world, rank, local, pg = bench.dist_setup(backend="gloo")
bench.barrier(pg)
slowest = bench.max_over_ranks(pg, 100.0 + 50.0 * rank, "cpu")
value = bench.aggregate_rate(world, 1000.0, 2, slowest)
bench.barrier(pg)
# the reference arm runs on rank 0 only; other ranks return without work
if rank != 0:
    assert bench.run_reference(None, world, rank, local, pg) is None
print(json.dumps({{"rank": rank, "world": world, "slowest": slowest, "value": value}}), flush=True)
pg.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_slowest_time(tmp_path):
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                   WORLD_SIZE="2", LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            pytest.fail("rank timed out")
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for r in outs:
        assert r["world"] == 2 and r["slowest"] == 150.0
        assert r["value"] == pytest.approx(2 * 1000.0 * 2 / 0.150)
