"""The multi-GPU form of bench.py (replicas only: one process per GPU, a gloo
group for the barrier and the max of the per-rank times) run as two CPU ranks
on 127.0.0.1: every rank takes the same collective steps and rank 0 gets the
slowest rank's time, as the job value requires."""
import os
import socket
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_PROGRAM = r"""
import os, sys, json
sys.path.insert(0, os.environ["REPO"])
import bench
d = bench.Dist(2)
d.barrier()
local = 1.5 + 2.0 * d.rank          # rank 1 is the slow one
worst = d.max(local)
d.barrier()
print(json.dumps({"rank": d.rank, "world": d.world, "max": worst}))
d.close()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_max():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, REPO=REPO, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_PROGRAM], env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=240) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, err[-2000:]
    import json
    lines = [json.loads(o.strip().splitlines()[-1]) for o, _ in outs]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    assert all(x["world"] == 2 and x["max"] == 3.5 for x in lines)
