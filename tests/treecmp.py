"""Comparison of the device tree/lists with the oracle's (test helper).

Boxes are identified by (level, centre): the device computes centres with
the reference's FP64 recursion, so equal boxes have bit-identical centres.
"""
import numpy as np


def _ids(level, centers):
    return [(int(l), tuple(np.asarray(c, dtype=np.float64).tolist())) for l, c in zip(level, centers)]


def compare(gpu, orc, check_lists=True, nlevend=None):
    """Returns a list of mismatch descriptions (empty = identical).

    List 1 is compared for target boxes at levels <= nlevend (the levels the
    direct loop visits, src/pfgt/pfgt.f:1087)."""
    bad = []
    if gpu["nlevels"] != orc["nlevels"]:
        bad.append(f"nlevels {gpu['nlevels']} != {orc['nlevels']}")
    if gpu["npwlevel"] != orc["npwlevel"]:
        bad.append(f"npwlevel {gpu['npwlevel']} != {orc['npwlevel']}")
    if gpu["bs0"] != orc["bs0"]:
        bad.append(f"bs0 {gpu['bs0']!r} != {orc['bs0']!r}")
    gid = _ids(gpu["level"], gpu["center"])
    oid = _ids(orc["ilevel"], orc["centers"])
    gmap = {k: i for i, k in enumerate(gid)}
    omap = {k: i for i, k in enumerate(oid)}
    if len(gmap) != len(gid):
        bad.append("duplicate device boxes")
    if set(gmap) != set(omap):
        only_g = len(set(gmap) - set(omap))
        only_o = len(set(omap) - set(gmap))
        bad.append(f"box sets differ: {only_g} only on device, {only_o} only in oracle "
                   f"(device {len(gmap)}, oracle {len(omap)})")
        return bad
    # per-box flags and point ranges
    for k, gi in gmap.items():
        oi = omap[k]
        if bool(gpu["nonleaf"][gi]) != (orc["nchild"][oi] > 0):
            bad.append(f"nonleaf differs at {k}")
            break
        if (gpu["src_lo"][gi] != orc["isrcse"][oi, 0] or
                gpu["src_hi"][gi] - gpu["src_lo"][gi] != orc["isrcse"][oi, 1] - orc["isrcse"][oi, 0] + 1):
            bad.append(f"source range differs at {k}")
            break
        if (gpu["trg_hi"][gi] - gpu["trg_lo"][gi] != orc["itrgse"][oi, 1] - orc["itrgse"][oi, 0] + 1):
            bad.append(f"target count differs at {k}")
            break
    if not np.array_equal(gpu["isrc"].astype(np.int64), orc["isrc"].astype(np.int64)):
        bad.append("source permutation differs")
    if not np.array_equal(gpu["itrg"].astype(np.int64), orc["itrg"].astype(np.int64)):
        bad.append("target permutation differs")
    if not check_lists:
        return bad
    # list 1 (as sets of source boxes per target box)
    nb = len(gid)
    for gi in range(nb):
        k = gid[gi]
        oi = omap[k]
        if nlevend is not None and k[0] > nlevend:
            continue
        gs = {gid[s] for s in gpu["l1_src"][gpu["l1_ptr"][gi]:gpu["l1_ptr"][gi + 1]]}
        os_ = {oid[s] for s in orc["list1"][oi, :orc["nlist1"][oi]]}
        if gs != os_:
            bad.append(f"list1 differs at box {k}: device {len(gs)} oracle {len(os_)}")
            break
    # plane-wave boxes
    nc = max(orc["npwlevel"], 0)
    if orc["npwlevel"] < orc["nlevels"]:
        lo, hi = orc["laddr"][nc]
        o_form = {oid[b] for b in range(lo, hi + 1)
                  if orc["isrcse"][b, 1] - orc["isrcse"][b, 0] + 1 > orc["ndiv"]}
        o_eval = {oid[b] for b in range(lo, hi + 1) if orc["ifpwexp"][b]}
        g_form = {gid[b] for b in gpu["form_box"]}
        g_eval = {gid[b] for b in gpu["eval_box"]}
        if o_form != g_form:
            bad.append(f"form boxes differ ({len(g_form)} vs {len(o_form)})")
        if o_eval != g_eval:
            bad.append(f"eval boxes differ ({len(g_eval)} vs {len(o_eval)})")
        if o_form == g_form and o_eval == g_eval:
            form_ids = [gid[b] for b in gpu["form_box"]]
            for e, b in enumerate(gpu["eval_box"]):
                k = gid[b]
                oi = omap[k]
                gl = {form_ids[s] for s in gpu["trans_src"][gpu["trans_ptr"][e]:gpu["trans_ptr"][e + 1]]}
                ol = {oid[s] for s in orc["listpw"][oi, :orc["nlistpw"][oi]]}
                if gl != ol:
                    bad.append(f"PW list differs at {k}")
                    break
    return bad
