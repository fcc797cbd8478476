"""The multi-rank logic of bench.py on CPU: two gloo ranks (no GPU).

bench.py shards grains across ranks (each rank its own seeded batch, weak
scaling, no data-path collective) and reduces the step time with a max over
ranks; the reference arm runs on rank 0 only.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, %(root)r)
import bench
rank = int(os.environ["RANK"])
d = bench.Dist(2, rank, backend="gloo")
d.barrier()
v = d.max(float(10 * rank + 3))
r, lam, m, dd = bench.grains(16, bench.rank_seed(rank))
d.barrier()
d.close()
print(json.dumps({"rank": rank, "max": v, "r0": float(r[0]), "d0": float(dd[0])}))
"""


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks():
    port = _port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD % {"root": ROOT}],
                                      env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda o: o["rank"])
    # max over ranks seen by both
    assert outs[0]["max"] == outs[1]["max"] == 13.0
    # disjoint grain sets per rank
    assert outs[0]["r0"] != outs[1]["r0"] and outs[0]["d0"] != outs[1]["d0"]


def test_reference_arm_rank1_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                        "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
