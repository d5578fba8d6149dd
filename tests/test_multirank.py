"""World-size-2 gloo test of the multi-rank plumbing on CPU: instances are
sharded across ranks with no data-path collective, results are identical to
the single-rank run, and the timing reduction is the max over ranks."""
import os
import socket
import subprocess
import sys

import numpy as np

from conftest import ROOT

CHILD = r"""
import os, sys, time, numpy as np
sys.path.insert(0, %(root)r)
import torch, torch.distributed as dist
from fgt_b200 import distributed as D, workloads as W
from oracle import oracle as O
rank, world = D.init(backend="gloo", timeout_s=60)
insts = W.batch_instances(count=6, nmin=200, nmax=800)
mine = D.shard_by_weight([x["sources"].shape[0] for x in insts], rank, world)
res = {}
t0 = time.perf_counter()
for i in mine:
    x = insts[i]
    r = O.pfgt(1, 3, x["delta"], x["eps"], 0, x["sources"], charge=x["charge"], ifpgh=1)
    res[i] = r["pot"]
dt = time.perf_counter() - t0
tmax = D.max_over_ranks(dt)
npts = D.sum_over_ranks(sum(insts[i]["sources"].shape[0] for i in mine))
assert tmax >= dt
assert npts == sum(x["sources"].shape[0] for x in insts)
np.savez(os.path.join(%(out)r, "rank%%d.npz" %% rank), **{str(k): v for k, v in res.items()})
dist.barrier()
dist.destroy_process_group()
print("rank", rank, "ok")
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_sharding(tmp_path, oracle):
    code = CHILD % {"root": ROOT, "out": str(tmp_path)}
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=300)[0] for p in procs]
    for p, o in zip(procs, outs):
        assert p.returncode == 0, o
    from fgt_b200 import distributed as D, workloads as W
    insts = W.batch_instances(count=6, nmin=200, nmax=800)
    got = {}
    for r in range(2):
        d = np.load(tmp_path / ("rank%d.npz" % r))
        got.update({int(k): d[k] for k in d.files})
    assert sorted(got) == list(range(6))
    for i, x in enumerate(insts):
        ref = oracle.pfgt(1, 3, x["delta"], x["eps"], 0, x["sources"], charge=x["charge"],
                          ifpgh=1)
        np.testing.assert_array_equal(got[i], ref["pot"])
    # shard helpers cover every item exactly once
    for n in (0, 1, 7, 64):
        spans = [D.shard(n, r, 3) for r in range(3)]
        assert sum(hi - lo for lo, hi in spans) == n
