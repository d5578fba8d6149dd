"""Multi-GPU pfgt: one process per GPU over torch.distributed.

Two ways to use several GPUs:

* independent problems (instances of a batch, replicas of one workload)
  shard by problem with no data-path collective (`shard`, `shard_by_weight`);
* one large point set shards *spatially* (`pfgt_sharded`): every rank passes
  its own part of the sources and targets and gets back the outputs of those
  points.

Spatial sharding follows from the structure of pfgt (src/pfgt/pfgt.f:6-409):
every interaction of a point, plane-wave or direct, comes from the 3^dim
boxes of the cut-off level around the point's box (the plane-wave lists and
list 1 are built from colleagues at that level, src/common/tree_routs_nd.f:
1063-1555, and the direct sums are truncated at sqrt(delta*log(1/eps)), the
side of a cut-off box, src/pfgt/pfgt.f:1084).  So:

1. the ranks agree on the root box and the cut-off level of the whole point
   set (an all-reduce of the bounding box, then the scalar formulas of
   pts_tree_boxsize0, src/common/pts_tree_nd.f:1330-1414, on the host);
2. the occupied cut-off boxes, in Morton order and weighted by their points,
   are cut into contiguous ranges of equal weight, one per rank;
3. every point moves to the rank owning its box, and every source also to
   the ranks owning one of its box's neighbours (a one-box halo);
4. each rank runs pfgt on its owned sources + halo sources and its owned
   targets with the whole set's root box (`root_level`), keeping the owned
   outputs;
5. the outputs go back to the ranks the points came from.

Step 4 builds each rank's tree from the points it holds: boxes above the
cut-off level may refine differently from the single-rank tree, which changes
how (plane waves or direct sums), not which, sources are added; results
agree with the single-rank call to the requested precision.  The exchanges
are all-to-all collectives over the process group (NCCL between GPUs, gloo
on the host).
"""
import datetime
import math
import os

import numpy as np


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=120):
    """Initialise the process group when launched by torchrun (world > 1)."""
    import torch.distributed as dist
    rank, world, _ = env_rank()
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world


def shard(n_items, rank, world):
    """Contiguous, balanced share [lo, hi) of n_items for `rank`."""
    base, rem = divmod(n_items, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def shard_by_weight(weights, rank, world):
    """Greedy longest-first assignment of weighted items to ranks; returns the
    item indices of `rank` (deterministic, identical on every rank)."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += weights[i]
    return [i for i in range(len(weights)) if owner[i] == rank]


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------ spatial sharding
def root_geometry(dim, delta, eps, iperiod, lo, hi, bs0=1.0, cen0=None):
    """Root box and cut-off level of pts_tree_boxsize0
    (src/common/pts_tree_nd.f:1330-1414) from the bounding box [lo, hi] of
    the whole point set (free space), or from the given bs0/cen0 (periodic).
    Returns (bs0, cen0, npwlevel) with the library's FP64 arithmetic."""
    if iperiod != 1:
        lo = np.asarray(lo, dtype=np.float64)
        hi = np.asarray(hi, dtype=np.float64)
        bs0 = float(np.max(hi - lo))
        cen0 = (lo + hi) / 2
    else:
        cen0 = np.zeros(dim) if cen0 is None else np.asarray(cen0, dtype=np.float64)[:dim]
    dc = math.sqrt(delta * math.log(1.0 / eps))
    levcut = int(math.log(bs0 / dc) / math.log(2.0))  # Fortran int(): toward zero
    if iperiod != 1 and bs0 >= dc:
        levcut += 1
        bs0 = math.ldexp(1.0, levcut) * dc
    return bs0, np.asarray(cen0, dtype=np.float64), levcut


def cutoff_coords(x, bs0, cen0, level):
    """Integer coordinates of every point's box at `level` by the tree's FP64
    centre recursion (x - c >= 0 picks the upper child, c moves by
    boxsize(l+1)/2; src/common/pts_tree_nd.f:733-737), so the assignment is
    that of the device tree."""
    x = np.asarray(x, dtype=np.float64)
    n, dim = x.shape
    c = np.broadcast_to(np.asarray(cen0, dtype=np.float64)[:dim], (n, dim)).copy()
    ic = np.zeros((n, dim), dtype=np.int64)
    bs = bs0
    for _ in range(max(level, 0)):
        bsc = bs / 2
        h = bsc / 2
        up = (x - c) >= 0
        ic = 2 * ic + up
        c = c + np.where(up, h, -h)
        bs = bsc
    return ic


def morton(ic, level):
    """Key of integer box coordinates at `level`: digits of `dim` bits per
    level, bit k set for the upper half in dimension k, coarsest first (the
    order of the tree's path keys)."""
    ic = np.asarray(ic, dtype=np.int64)
    n, dim = ic.shape
    key = np.zeros(n, dtype=np.int64)
    for j in range(level - 1, -1, -1):
        dig = np.zeros(n, dtype=np.int64)
        for k in range(dim):
            dig |= ((ic[:, k] >> j) & 1) << k
        key = (key << dim) | dig
    return key


def partition(keys, weights, world):
    """Cut occupied boxes (sorted unique keys with weights) into `world`
    contiguous key ranges of about equal weight; returns the first key of
    every rank's range (starts[0] = 0 means: every smaller key is rank 0's)."""
    keys = np.asarray(keys, dtype=np.int64)
    w = np.asarray(weights, dtype=np.float64)
    starts = np.zeros(world, dtype=np.int64)
    if len(keys) == 0:
        return starts
    cum = np.cumsum(w)
    tot = cum[-1]
    for r in range(1, world):
        i = int(np.searchsorted(cum, tot * r / world, side="left"))
        i = min(max(i + 1, 0), len(keys))
        starts[r] = keys[i] if i < len(keys) else keys[-1] + 1
    return np.maximum.accumulate(starts)


def owner_of(keys, starts):
    """Rank owning each key (the last range start not above it)."""
    return np.searchsorted(starts, np.asarray(keys, dtype=np.int64), side="right") - 1


def neighbour_owners(ic, level, iperiod, occupied, starts):
    """For every point (box coordinates ic at `level`), the set of ranks that
    own an occupied box among the 3^dim boxes around it (the box itself
    included), as a boolean matrix [n, world].  Periodic: neighbours wrap."""
    ic = np.asarray(ic, dtype=np.int64)
    n, dim = ic.shape
    world = len(starts)
    nb = 1 << max(level, 0)
    out = np.zeros((n, world), dtype=bool)
    occupied = np.asarray(occupied, dtype=np.int64)
    for off in np.ndindex(*([3] * dim)):
        q = ic + (np.asarray(off) - 1)
        if iperiod == 1:
            q = np.mod(q, nb)
            ok = np.ones(n, dtype=bool)
        else:
            ok = np.all((q >= 0) & (q < nb), axis=1)
        qk = morton(np.where(ok[:, None], q, 0), level)
        pos = np.searchsorted(occupied, qk)
        occ = ok & (pos < len(occupied)) & (occupied[np.minimum(pos, len(occupied) - 1)] == qk)
        r = owner_of(qk, starts)
        out[np.nonzero(occ)[0], r[occ]] = True
    return out


def _exchange(blocks, group=None):
    """All-to-all of float64 row blocks: blocks[r] goes to rank r; returns the
    blocks received from every rank (same column count everywhere)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    ncol = blocks[0].shape[1]
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else "cpu"
    send_n = torch.tensor([b.shape[0] for b in blocks], dtype=torch.int64, device=dev)
    recv_n = torch.empty(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_n, send_n, group=group)
    rn = recv_n.cpu().numpy().tolist()
    sn = send_n.cpu().numpy().tolist()
    send = torch.from_numpy(np.concatenate(blocks).reshape(-1)).to(dev)
    recv = torch.empty(sum(rn) * ncol, dtype=torch.float64, device=dev)
    dist.all_to_all_single(recv, send, [r * ncol for r in rn], [s * ncol for s in sn],
                           group=group)
    flat = recv.cpu().numpy().reshape(-1, ncol)
    out, o = [], 0
    for r in rn:
        out.append(flat[o:o + r])
        o += r
    return out


def pfgt_sharded(nd, dim, delta, eps, iperiod, sources, charge=None, dipstr=None,
                 rnormal=None, ifpgh=1, targets=None, ifpghtarg=0, bs0=1.0, cen0=None,
                 local_solver=None, group=None, **solver_kw):
    """Spatially sharded pfgt over the ranks of `group`: this rank's sources
    (ns_r, dim), strengths and targets in, this rank's outputs out (the dict
    of `fgt_b200.pfgt`, rows in this rank's input order).  Every rank must
    call it.  local_solver(**pfgt arguments) runs one rank's share (default:
    `fgt_b200.pfgt` on this process's GPU); it must accept root_level."""
    import torch
    import torch.distributed as dist
    if local_solver is None:
        import fgt_b200
        local_solver = fgt_b200.pfgt
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    src = np.ascontiguousarray(sources, dtype=np.float64).reshape(-1, dim)
    trg = (np.zeros((0, dim)) if targets is None
           else np.ascontiguousarray(targets, dtype=np.float64).reshape(-1, dim))
    ns, nt = src.shape[0], trg.shape[0]
    if nt == 0:
        ifpghtarg = 0
    # 1. root box and cut-off level of the whole set
    pts = np.concatenate([src, trg])
    lo = pts.min(axis=0) if len(pts) else np.full(dim, np.inf)
    hi = pts.max(axis=0) if len(pts) else np.full(dim, -np.inf)
    bb = torch.from_numpy(np.concatenate([-lo, hi]))
    dist.all_reduce(bb, op=dist.ReduceOp.MAX, group=group)
    bb = bb.numpy()
    g_bs0, g_cen0, level = root_geometry(dim, delta, eps, iperiod, -bb[:dim], bb[dim:], bs0,
                                         cen0)
    lev = max(level, 0)
    # 2. occupied cut-off boxes and their weights, merged over the ranks
    sic, tic = cutoff_coords(src, g_bs0, g_cen0, lev), cutoff_coords(trg, g_bs0, g_cen0, lev)
    skey, tkey = morton(sic, lev), morton(tic, lev)
    k, cnt = np.unique(np.concatenate([skey, tkey]), return_counts=True)
    allk = [None] * world
    dist.all_gather_object(allk, (k, cnt), group=group)
    keys = np.concatenate([a for a, _ in allk])
    ws = np.concatenate([b for _, b in allk]).astype(np.float64)
    occupied, inv = np.unique(keys, return_inverse=True)
    wsum = np.zeros(len(occupied))
    np.add.at(wsum, inv, ws)
    starts = partition(occupied, wsum, world)
    # 3. route: sources to their owner and to the owners of neighbouring boxes
    s_owner = owner_of(skey, starts)
    ubox, first, binv = np.unique(skey, return_index=True, return_inverse=True)
    s_dest = neighbour_owners(sic[first], lev, iperiod, occupied, starts)[binv.reshape(-1)]
    t_owner = owner_of(tkey, starts)
    ifcharge, ifdipole = charge is not None, dipstr is not None
    cols = [src]
    if ifcharge:
        cols.append(np.ascontiguousarray(charge, dtype=np.float64).reshape(ns, nd))
    if ifdipole:
        cols.append(np.ascontiguousarray(dipstr, dtype=np.float64).reshape(ns, nd))
        cols.append(np.ascontiguousarray(rnormal, dtype=np.float64).reshape(ns, dim))
    idx = np.arange(ns, dtype=np.float64)[:, None]
    srow = np.concatenate(cols + [idx, np.zeros((ns, 1))], axis=1)
    sblocks = []
    for r in range(world):
        own = s_owner == r
        halo = s_dest[:, r] & ~own
        a = srow[own].copy()
        a[:, -1] = 1.0  # owned here: its outputs go back
        b = srow[halo].copy()
        sblocks.append(np.concatenate([a, b]))
    trow = np.concatenate([trg, np.arange(nt, dtype=np.float64)[:, None]], axis=1)
    tblocks = [trow[t_owner == r] for r in range(world)]
    s_in = _exchange(sblocks, group)
    t_in = _exchange(tblocks, group)
    # 4. this rank's share: owned sources first, then the halo
    S = np.concatenate(s_in)
    S = np.concatenate([S[S[:, -1] == 1.0], S[S[:, -1] != 1.0]])
    n_own = int(np.sum(S[:, -1] == 1.0))
    T = np.concatenate(t_in)
    c = dim
    kw = dict(solver_kw)
    if ifcharge:
        kw["charge"] = S[:, c:c + nd]
        c += nd
    if ifdipole:
        kw["dipstr"] = S[:, c:c + nd]
        kw["rnormal"] = S[:, c + nd:c + nd + dim]
    nh = dim * (dim + 1) // 2
    fields_s = [("pot", nd)] + ([("grad", dim * nd)] if ifpgh >= 2 else []) + \
               ([("hess", nh * nd)] if ifpgh >= 3 else [])
    fields_t = [("pottarg", nd)] + ([("gradtarg", dim * nd)] if ifpghtarg >= 2 else []) + \
               ([("hesstarg", nh * nd)] if ifpghtarg >= 3 else [])
    fields_s = fields_s if ifpgh >= 1 else []
    fields_t = fields_t if ifpghtarg >= 1 else []
    res = {}
    if S.shape[0] > 0 and (n_own > 0 or T.shape[0] > 0):
        res = local_solver(nd=nd, dim=dim, delta=delta, eps=eps, iperiod=iperiod,
                           sources=S[:, :dim], ifpgh=ifpgh if n_own else 0,
                           targets=T[:, :dim] if T.shape[0] else None,
                           ifpghtarg=ifpghtarg if T.shape[0] else 0, bs0=g_bs0, cen0=g_cen0,
                           root_level=level if iperiod != 1 else -1, **kw)
    # 5. outputs back to the ranks the points came from
    def back(meta_idx, fields, n_local, rows_of):
        # outputs of this rank's owned points with their origin indices
        w_all = sum(w for _, w in fields)
        if n_local == 0:
            return np.zeros((0, w_all + 1))
        parts = [np.asarray(res[f]).reshape(-1, w)[rows_of] if f in res
                 else np.zeros((n_local, w)) for f, w in fields]
        return np.concatenate(parts + [meta_idx[:, None]], axis=1)

    so = back(S[:n_own, -2], fields_s, n_own, slice(0, n_own))
    to = back(T[:, -1], fields_t, T.shape[0], slice(0, T.shape[0]))
    # owned rows are sent back to their origin: origin rank per received block
    s_orig, t_orig = [], []
    for r, blk in enumerate(s_in):
        s_orig.append(np.full(int(np.sum(blk[:, -1] == 1.0)), r))
    for r, blk in enumerate(t_in):
        t_orig.append(np.full(blk.shape[0], r))
    s_orig = np.concatenate(s_orig) if s_orig else np.zeros(0, dtype=np.int64)
    t_orig = np.concatenate(t_orig) if t_orig else np.zeros(0, dtype=np.int64)
    s_back = _exchange([so[s_orig == r] for r in range(world)], group)
    t_back = _exchange([to[t_orig == r] for r in range(world)], group)
    out = {"bs0": g_bs0, "cen0": g_cen0, "npwlevel": level}
    for fields, back_rows, n, shape_of in (
            (fields_s, s_back, ns, lambda f: {"pot": (nd,), "grad": (dim, nd), "hess": (nh, nd)}[f]),
            (fields_t, t_back, nt, lambda f: {"pottarg": (nd,), "gradtarg": (dim, nd),
                                              "hesstarg": (nh, nd)}[f])):
        if not fields:
            continue
        rows = np.concatenate(back_rows)
        order = rows[:, -1].astype(np.int64)
        c = 0
        for f, w in fields:
            a = np.zeros((n, w))
            a[order] = rows[:, c:c + w]
            out[f] = a.reshape((n,) + shape_of(f))
            c += w
    return out
