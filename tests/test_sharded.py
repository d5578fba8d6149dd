"""Spatial sharding of one pfgt over ranks (fgt_b200.distributed.pfgt_sharded),
tested on the host: the partition and one-box halo logic with numpy, and the
whole exchange with two gloo ranks whose per-rank share is computed by the
oracle (the GPU library takes that role on GPUs).  The reassembled outputs
must equal the single-rank result to the requested precision."""
import math
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, relerr
from fgt_b200 import distributed as D
from fgt_b200 import workloads as W


def test_root_geometry_matches_the_restatement(oracle):
    rng = np.random.default_rng(1)
    x = W.gaussian_clusters(rng, 3000, 3, ncl=5)
    t = oracle.tree(3, 1e-4, 1e-6, 0, x, np.zeros((0, 3)))
    bs0, cen0, lev = D.root_geometry(3, 1e-4, 1e-6, 0, x.min(axis=0), x.max(axis=0))
    assert bs0 == t["bs0"] and lev == t["npwlevel"]
    np.testing.assert_array_equal(cen0, t["cen0"])


def test_cutoff_boxes_match_the_tree(oracle):
    """Box coordinates from the host recursion equal the restatement's tree
    boxes at the cut-off level (same FP64 centre recursion)."""
    rng = np.random.default_rng(2)
    x = W.uniform(rng, 4000, 2)
    t = oracle.tree(2, 1e-3, 1e-6, 0, x, np.zeros((0, 2)))
    bs0, cen0, lev = D.root_geometry(2, 1e-3, 1e-6, 0, x.min(axis=0), x.max(axis=0))
    ic = D.cutoff_coords(x, bs0, cen0, lev)
    h = bs0 / 2 ** lev
    centres = cen0 - bs0 / 2 + (ic + 0.5) * h
    # every point lies in its box (the boundary goes to the upper box)
    assert np.all(x - (centres - h / 2) >= 0) and np.all(x - (centres + h / 2) < 1e-15)
    # every point's leaf in the tree agrees with its cut-off box: a finer
    # leaf lies inside the box, a coarser (or equal) leaf contains it
    leaves = np.nonzero(t["nchild"] == 0)[0]
    for b in leaves:
        s0, s1 = t["isrcse"][b]
        if s1 < s0:
            continue
        pts = t["isrc"][s0:s1 + 1]
        lb = t["ilevel"][b]
        hb = bs0 / 2 ** lb
        cb = np.round((t["centers"][b] - (cen0 - bs0 / 2)) / hb - 0.5).astype(np.int64)
        if lb >= lev:
            np.testing.assert_array_equal(ic[pts], np.broadcast_to(cb >> (lb - lev), ic[pts].shape))
        else:
            np.testing.assert_array_equal(ic[pts] >> (lev - lb), np.broadcast_to(cb, ic[pts].shape))


@pytest.mark.parametrize("iperiod", [0, 1])
@pytest.mark.parametrize("world", [2, 3, 5])
def test_partition_and_halo_cover_every_interaction(iperiod, world):
    """Every source within the cut-off distance of a rank's owned point is on
    that rank (owned or halo), and every occupied box has one owner."""
    rng = np.random.default_rng(10 + world)
    dim, delta, eps = 2, 1e-3, 1e-6
    x = np.concatenate([W.uniform(rng, 3000, dim), W.gaussian_clusters(rng, 3000, dim, ncl=3)])
    if iperiod:
        x = np.mod(x + 0.5, 1.0) - 0.5
        bs0, cen0, lev = D.root_geometry(dim, delta, eps, 1, None, None, 1.0, [0.0, 0.0])
    else:
        bs0, cen0, lev = D.root_geometry(dim, delta, eps, 0, x.min(axis=0), x.max(axis=0))
    ic = D.cutoff_coords(x, bs0, cen0, lev)
    key = D.morton(ic, lev)
    occ, cnt = np.unique(key, return_counts=True)
    starts = D.partition(occ, cnt, world)
    own = D.owner_of(key, starts)
    loads = np.bincount(own, minlength=world)
    assert loads.sum() == len(x) and loads.max() <= 2.0 * len(x) / world + cnt.max()
    dest = D.neighbour_owners(ic, lev, iperiod, occ, starts)
    assert np.all(dest[np.arange(len(x)), own])  # a box's owner gets its sources
    dc = math.sqrt(delta * math.log(1 / eps))
    for r in range(world):
        mine = np.nonzero(own == r)[0]
        have = dest[:, r]
        for i in mine[:: max(1, len(mine) // 200)]:
            d = x - x[i]
            if iperiod:
                d = d - np.round(d / bs0) * bs0
            near = np.nonzero(np.sum(d * d, axis=1) < dc * dc)[0]
            assert have[near].all(), (r, i)


CHILD = r"""
import os, sys, numpy as np
sys.path.insert(0, %(root)r)
import torch.distributed as dist
from fgt_b200 import distributed as D
from oracle import oracle as O
rank, world = D.init(backend="gloo", timeout_s=120)
d = np.load(%(inp)r)
mine = d["owner"] == rank
tmine = d["towner"] == rank
kw = dict(nd=int(d["nd"]), dim=int(d["dim"]), delta=float(d["delta"]), eps=float(d["eps"]),
          iperiod=int(d["iperiod"]), bs0=1.0, cen0=[0.0] * int(d["dim"]))
trg = d["trg"][tmine] if d["trg"].shape[0] else None
r = D.pfgt_sharded(sources=d["src"][mine], charge=d["q"][mine], ifpgh=2, targets=trg,
                   ifpghtarg=2 if trg is not None else 0,
                   local_solver=lambda **a: O.pfgt(**a), **kw)
np.savez(os.path.join(%(out)r, "rank%%d.npz" %% rank), **{k: v for k, v in r.items()
                                                         if isinstance(v, np.ndarray)})
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


CASES = [
    ("2d_free", dict(nd=1, dim=2, delta=1e-3, eps=1e-6, iperiod=0), 8000, 1500),
    ("2d_periodic_nd2", dict(nd=2, dim=2, delta=1e-3, eps=1e-6, iperiod=1), 8000, 0),
    ("3d_free_clusters", dict(nd=1, dim=3, delta=3e-3, eps=1e-6, iperiod=0), 5000, 500),
]


@pytest.mark.parametrize("name,geo,ns,nt", CASES, ids=[c[0] for c in CASES])
def test_two_rank_sharded_pfgt_matches_single_rank(tmp_path, oracle, name, geo, ns, nt):
    rng = np.random.default_rng(7)
    dim, nd = geo["dim"], geo["nd"]
    src = W.gaussian_clusters(rng, ns, dim, ncl=4) if dim == 3 else W.uniform(rng, ns, dim)
    q = rng.uniform(-1, 1, (ns, nd))
    trg = W.uniform(rng, nt, dim) if nt else np.zeros((0, dim))
    # each rank starts with an arbitrary share of the points (not spatial)
    owner = rng.integers(0, 2, ns)
    towner = rng.integers(0, 2, nt)
    inp = str(tmp_path / "in.npz")
    np.savez(inp, src=src, q=q, trg=trg, owner=owner, towner=towner, **geo)
    code = CHILD % {"root": ROOT, "out": str(tmp_path), "inp": inp}
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=600)[0] for p in procs]
    for p, o in zip(procs, outs):
        assert p.returncode == 0, o
    ref = oracle.pfgt(sources=src, charge=q, ifpgh=2, targets=trg if nt else None,
                      ifpghtarg=2 if nt else 0, bs0=1.0, cen0=[0.0] * dim, **geo)
    got = {}
    for r in range(2):
        d = np.load(tmp_path / ("rank%d.npz" % r))
        m, tm = owner == r, towner == r
        for f in ("pot", "grad"):
            got.setdefault(f, np.zeros_like(ref[f]))[m] = d[f]
        if nt:
            for f in ("pottarg", "gradtarg"):
                got.setdefault(f, np.zeros_like(ref[f]))[tm] = d[f]
    for f in got:
        e = relerr(ref[f], got[f])
        assert e < geo["eps"], (name, f, e)


@pytest.mark.gpu
def test_root_level_option_reproduces_the_free_space_call(fgt):
    """The library with the root box given (root_level) builds the tree the
    free-space call builds from the points: same outputs."""
    rng = np.random.default_rng(4)
    x = W.gaussian_clusters(rng, 20000, 3, ncl=6)
    q = rng.uniform(-1, 1, (20000, 1))
    kw = dict(nd=1, dim=3, delta=3e-3, eps=1e-6, iperiod=0, sources=x, charge=q, ifpgh=2,
              precision=fgt.PREC_FP64)
    a = fgt.pfgt(**kw)
    bs0, cen0, lev = D.root_geometry(3, 3e-3, 1e-6, 0, x.min(axis=0), x.max(axis=0))
    assert bs0 == a["bs0"]
    b = fgt.pfgt(bs0=bs0, cen0=cen0, root_level=lev, stats=True, **kw)
    assert b["stats"]["npwlevel"] == lev and b["stats"]["n_form_boxes"] > 0
    # same tree; the spreading's shared-memory atomics add in a run-dependent order
    assert relerr(a["pot"], b["pot"]) < 1e-12
    assert relerr(a["grad"], b["grad"]) < 1e-12


@pytest.mark.gpu
def test_sharded_call_on_one_gpu_rank(fgt, tmp_path):
    """pfgt_sharded with the GPU library as the per-rank solver, one rank
    (the exchanges degenerate; the root box and routing logic still run)."""
    import torch.distributed as dist
    store = dist.FileStore(str(tmp_path / "store"), 1)
    dist.init_process_group("gloo", store=store, rank=0, world_size=1)
    try:
        rng = np.random.default_rng(6)
        x = W.sphere_surface(rng, 30000, radius=0.35)
        t = W.uniform(rng, 3000, 3)
        q = rng.uniform(-1, 1, (30000, 1))
        kw = dict(nd=1, dim=3, delta=1e-3, eps=1e-6, iperiod=0, charge=q, ifpgh=2,
                  targets=t, ifpghtarg=2)
        r = D.pfgt_sharded(sources=x, precision=fgt.PREC_FP64, **kw)
        ref = fgt.pfgt(sources=x, precision=fgt.PREC_FP64, **kw)
        for f in ("pot", "grad", "pottarg", "gradtarg"):
            assert relerr(ref[f], r[f]) < 1e-12, f
    finally:
        dist.destroy_process_group()
