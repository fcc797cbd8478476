"""get_table over several ranks (costuum_b200/shard.py): every rank computes
the grid for its own sizes (round robin over the ascending sizes), and the
gathered table is placed back by size.

* CPU: the partition covers every size exactly once and the merge inverts
  it; two gloo ranks run shard.get_table with the per-rank computation
  replaced by a deterministic stand-in that depends on the cell alone, and
  both ranks return the table a single process returns.
* GPU: two gloo ranks on one GPU (each its own context; nothing in one
  rank's kernels waits on the other) compute a Draine-Hensley grid with
  alignment, extinction, absorption and scattering matrices; the gathered
  table equals the one-process get_table bit for bit.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_and_merge():
    from costuum_b200 import shard
    for nsizes in (1, 2, 5, 8):
        for world in (1, 2, 3, 4):
            idx = np.concatenate([shard.size_shard(nsizes, world, r)
                                  for r in range(world)])
            assert np.array_equal(np.sort(idx), np.arange(nsizes))
            full = np.random.default_rng(nsizes).standard_normal((2, nsizes, 3, 4))
            parts = [full[:, shard.size_shard(nsizes, world, r)] for r in range(world)]
            assert np.array_equal(shard.merge_shards(parts, nsizes, world, 1), full)


FAKE_CHILD = r"""
import json, os, sys
sys.path.insert(0, %(root)r)
import numpy as np
import torch.distributed as dist
from costuum_b200 import CosTuuM, shard

def fake(types, sizes, lams, thetas, shp, al, dust, return_status=False, **kw):
    # a value that depends on the cell alone, as a real get_table's does
    t = np.asarray(types)[:, None, None, None, None]
    s = np.asarray(sizes)[None, :, None, None, None]
    l = np.asarray(lams)[None, None, :, None, None]
    th = np.asarray(thetas)[None, None, None, :, None]
    k = np.arange(5)[None, None, None, None, :]
    q = np.sin(t + 1e6 * s) * np.cos(1e6 * l + th) + k
    st = np.zeros((len(types), len(sizes), len(lams), len(shp.shapes)), np.int32)
    return (q, st) if return_status else q

CosTuuM.get_table = fake
dist.init_process_group("gloo")
sizes = np.array([0.9, 0.1, 0.5, 0.3, 0.7]) * 1e-6
shp = CosTuuM.SingleShapeShapeDistribution(2.0)
q = shard.get_table([0, 1], sizes, [1e-6, 2e-6], [0.1, 0.7, 1.3], shp, None, None,
                    do_extinction=True)
ref = fake(np.array([0, 1]), np.sort(sizes), [1e-6, 2e-6], [0.1, 0.7, 1.3], shp,
           None, None)
ok = bool(np.array_equal(q, ref))
dist.destroy_process_group()
print(json.dumps({"rank": int(os.environ["RANK"]), "ok": ok}))
"""


def _run_ranks(code, world=2, timeout=300):
    port = _port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world),
                   LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=timeout)
        assert p.returncode == 0, err[-3000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    return outs


def test_two_gloo_ranks_gather_the_table():
    outs = _run_ranks(FAKE_CHILD % {"root": ROOT})
    assert all(o["ok"] for o in outs)


GPU_CHILD = r"""
import json, os, sys
sys.path.insert(0, %(root)r)
import numpy as np
import torch.distributed as dist
from costuum_b200 import CosTuuM as C, shard

dist.init_process_group("gloo")
kw = dict(types=np.array([0]), sizes=np.array([0.05e-6, 0.3e-6, 0.12e-6, 0.6e-6, 0.2e-6]),
          wavelengths=np.array([1.5e-6, 0.8e-6]), thetas=np.array([0.3, 1.2, 2.0]),
          shape_distribution=C.DraineHensleyShapeDistribution(4),
          alignment_distribution=C.SizeBasedAlignmentDistribution(
              0.1e-6, C.MISHCHENKO_ALIGNMENT, maximum_order=30),
          dust_properties=C.CustomDustProperties(
              lambda w, s, t: (1.4 + 0.3 * s / 1e-6) + 0.05j * (1e-6 / w)),
          maximum_order=30, do_extinction=True, do_scattering=True)
q, z, st = shard.get_table(return_status=True, **kw)
out = {"rank": int(os.environ["RANK"])}
if out["rank"] == 0:
    q1, z1 = C.get_table(**kw)
    out["q_equal"] = bool(np.array_equal(q.reshape(q1.shape), q1))
    out["z_equal"] = bool(np.array_equal(z.reshape(z1.shape), z1))
    out["status_ok"] = bool((st == 0).all())
dist.destroy_process_group()
print(json.dumps(out))
"""


@pytest.mark.gpu
def test_two_ranks_on_one_gpu_bitwise():
    outs = _run_ranks(GPU_CHILD % {"root": ROOT}, timeout=600)
    r0 = [o for o in outs if o["rank"] == 0][0]
    assert r0["q_equal"] and r0["z_equal"] and r0["status_ok"], r0
