"""CPU tests of the oracle (the restatement of the reference pfgt).

The reference ships no golden vectors; the restatement is pinned against the
exact FP64 Gauss transform (the mathematical definition) with the accuracy
criterion of the reference's own test driver (test/pfgt/test_pfgt_all.f:
437-512, relative l2 error per field), against the reference test's special
point scenarios, and against committed fixtures (tests/golden/).
"""
import os

import numpy as np
import pytest

from conftest import relerr
from fgt_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

CASES = [
    # dim, n, delta, eps, iperiod, ifpgh, nd, dipole, ntarg
    (2, 3000, 1e-3, 1e-6, 0, 2, 1, False, 0),
    (2, 3000, 1e-4, 1e-6, 0, 3, 1, False, 300),
    (3, 4000, 1e-3, 1e-6, 0, 2, 1, False, 0),
    (3, 20000, 1e-2, 1e-3, 0, 2, 1, False, 0),
    (2, 3000, 1e-3, 1e-6, 1, 2, 1, False, 0),
    (2, 3000, 3e-2, 1e-6, 1, 2, 1, False, 0),
    (2, 2000, 1e-3, 1e-6, 0, 3, 2, True, 300),
    (1, 2000, 1e-4, 1e-9, 0, 3, 1, False, 300),
    (2, 300, 10.0, 1e-6, 0, 2, 1, False, 0),
]


def _inputs(rng, dim, n, nd, dip, ntarg):
    src = W.uniform(rng, n, dim)
    q = rng.uniform(-1, 1, (n, nd))
    ds = rng.uniform(-1, 1, (n, nd)) if dip else None
    rn = rng.standard_normal((n, dim)) if dip else None
    trg = W.uniform(rng, ntarg, dim) if ntarg else None
    return src, q, ds, rn, trg


@pytest.mark.parametrize("case", CASES, ids=lambda c: "d%d_n%d_del%g_eps%g_per%d" % c[:5])
def test_oracle_vs_exact(oracle, case):
    dim, n, delta, eps, per, pgh, nd, dip, ntarg = case
    rng = np.random.default_rng(abs(hash(case)) % 2**32)
    src, q, ds, rn, trg = _inputs(rng, dim, n, nd, dip, ntarg)
    r = oracle.pfgt(nd, dim, delta, eps, per, src, charge=q, dipstr=ds, rnormal=rn,
                    ifpgh=pgh, targets=trg, ifpghtarg=pgh if ntarg else 0, bs0=1.0,
                    cen0=[0.0] * dim)
    idx = rng.choice(n, min(n, 60), replace=False)
    ex = oracle.direct_exact(nd, dim, delta, src, src[idx], charge=q, dipstr=ds, rnormal=rn,
                             ifpgh=pgh, iperiod=per, bs0=1.0)
    # truncation of the near field at delta*log(1/eps) bounds the accuracy
    assert relerr(ex["pot"], r["pot"][idx]) < 10 * eps
    if pgh >= 2:
        assert relerr(ex["grad"], r["grad"][idx]) < 30 * eps
    if pgh >= 3:
        assert relerr(ex["hess"], r["hess"][idx]) < 100 * eps
    if ntarg:
        tid = rng.choice(ntarg, min(ntarg, 60), replace=False)
        ext = oracle.direct_exact(nd, dim, delta, src, trg[tid], charge=q, dipstr=ds,
                                  rnormal=rn, ifpgh=pgh, iperiod=per, bs0=1.0)
        assert relerr(ext["pot"], r["pottarg"][tid]) < 10 * eps


@pytest.mark.parametrize("dim,n,delta,eps", [(2, 20000, 1e-4, 1e-6), (3, 20000, 1e-2, 1e-3),
                                             (1, 3000, 1e-4, 1e-9)])
def test_fast_nufft_matches_exact(oracle, dim, n, delta, eps):
    """The timed CPU baseline (ES-kernel NUFFT) agrees with the exact DFTs."""
    rng = np.random.default_rng(3)
    src = W.uniform(rng, n, dim)
    q = rng.uniform(-1, 1, (n, 1))
    a = oracle.pfgt(1, dim, delta, eps, 0, src, charge=q, ifpgh=2)
    b = oracle.pfgt(1, dim, delta, eps, 0, src, charge=q, ifpgh=2, nufft="spread")
    assert relerr(a["pot"], b["pot"]) < 0.2 * eps
    assert relerr(a["grad"], b["grad"]) < 0.2 * eps


def test_single_source_is_a_gaussian(oracle):
    """One unit charge: the transform is exp(-|t-s|^2/delta) inside the
    cut-off, zero beyond it (pfgt_direct.f:66-71 keeps rr < dmax)."""
    s = np.array([[0.1, -0.2, 0.05]])
    rng = np.random.default_rng(0)
    t = s + rng.uniform(-0.05, 0.05, (200, 3))
    delta, eps = 1e-3, 1e-6
    r = oracle.pfgt(1, 3, delta, eps, 0, s, charge=np.ones((1, 1)), ifpgh=1, targets=t,
                    ifpghtarg=2)
    rr = np.sum((t - s) ** 2, axis=1)
    ex = np.where(rr < delta * np.log(1 / eps), np.exp(-rr / delta), 0.0)
    np.testing.assert_allclose(r["pottarg"][:, 0], ex, rtol=1e-12, atol=1e-15)
    g = -2 / delta * (t - s) * ex[:, None]
    np.testing.assert_allclose(r["gradtarg"][:, :, 0], g, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(r["pot"][0, 0], 1.0)  # self term included


def test_cutoff_boundary(oracle):
    """Pairs just inside / outside rr = delta*log(1/eps)."""
    delta, eps = 1e-3, 1e-6
    dmax = delta * np.log(1 / eps)
    s = np.zeros((1, 2))
    t = np.array([[np.sqrt(dmax) * (1 - 1e-9), 0.0], [np.sqrt(dmax) * (1 + 1e-9), 0.0]])
    r = oracle.pfgt(1, 2, delta, eps, 0, s, charge=np.ones((1, 1)), ifpgh=1, targets=t,
                    ifpghtarg=1)
    assert r["pottarg"][0, 0] > 0.9 * eps
    assert r["pottarg"][1, 0] == 0.0


def test_reference_scenario_special_sources(oracle):
    """Wiggly-curve sources with the corner sources at 0 and 1 and a unit
    charge at 0.05 (test/pfgt/test_pfgt_all.f:146-206), checked like the
    reference driver on sampled sources and targets."""
    rng = np.random.default_rng(11)
    n, delta, eps = 6000, 1e-3, 1e-6
    src = W.wiggly_curve(rng, n, 2)
    q = rng.uniform(0, 1, (n, 1))
    q[0] = q[1] = 0.0
    q[2] = 1.0
    trg = rng.uniform(0, 1, (2000, 2))
    r = oracle.pfgt(1, 2, delta, eps, 0, src, charge=q, ifpgh=3, targets=trg, ifpghtarg=2)
    ex = oracle.direct_exact(1, 2, delta, src, src[:20], charge=q, ifpgh=3)
    assert relerr(ex["pot"], r["pot"][:20]) < 10 * eps
    ext = oracle.direct_exact(1, 2, delta, src, trg[:20], charge=q, ifpgh=2)
    assert relerr(ext["pot"], r["pottarg"][:20]) < 10 * eps


def test_periodic_face_pairs(oracle):
    """Periodicity: targets on opposite faces of the unit cell get equal
    fields (test/pfgt/test_pfgt_all.f:217-311, 452-461)."""
    rng = np.random.default_rng(5)
    n, delta, eps = 8000, 1e-3, 1e-6
    src = rng.uniform(0, 1, (n, 2))
    q = rng.uniform(0, 1, (n, 1))
    nx = 12
    h = 1.0 / (nx + 1)
    lo = [[-0.5 + i * h + 0.5, 0.0] for i in range(1, nx + 1)] + \
         [[0.0, -0.5 + i * h + 0.5] for i in range(1, nx + 1)]
    hi = [[p[0], 1.0] if p[1] == 0.0 and p[0] != 0.0 else [1.0, p[1]] for p in lo]
    trg = np.array(lo + hi)
    r = oracle.pfgt(1, 2, delta, eps, 1, src, charge=q, ifpgh=1, targets=trg, ifpghtarg=2,
                    bs0=1.0, cen0=[0.5, 0.5])
    half = len(lo)
    assert relerr(r["pottarg"][:half], r["pottarg"][half:]) < 10 * eps


def test_quirks_are_documented(oracle):
    """The reference's output defects reproduce only when requested."""
    rng = np.random.default_rng(2)
    n = 4000
    src = W.uniform(rng, n, 2)
    q = rng.uniform(-1, 1, (n, 1))
    trg = W.uniform(rng, 500, 2)
    kw = dict(charge=q, ifpgh=2, targets=trg, ifpghtarg=2)
    good = oracle.pfgt(1, 2, 1e-4, 1e-6, 0, src, **kw)
    bad = oracle.pfgt(1, 2, 1e-4, 1e-6, 0, src, quirks=1, **kw)
    ex = oracle.direct_exact(1, 2, 1e-4, src, trg[:50], charge=q, ifpgh=2)
    assert relerr(ex["pot"], good["pottarg"][:50]) < 1e-5
    # quirk 4: a root below half the cut-off with ns <= ndiv returns zeros
    small = W.uniform(rng, 50, 2) * 0.01
    z = oracle.pfgt(1, 2, 1.0, 1e-6, 0, small, charge=np.ones((50, 1)), ifpgh=1, quirks=4)
    f = oracle.pfgt(1, 2, 1.0, 1e-6, 0, small, charge=np.ones((50, 1)), ifpgh=1)
    assert np.all(z["pot"] == 0)
    assert np.all(f["pot"] > 1)
    assert bad is not None


def test_tree_invariants(oracle):
    rng = np.random.default_rng(9)
    src = W.gaussian_clusters(rng, 20000, 3)
    t = oracle.tree(3, 1e-5, 1e-9, 0, src, np.zeros((0, 3)))
    nb = t["nboxes"]
    leaf = t["nchild"] == 0
    # every point in exactly one leaf
    cnt = np.zeros(src.shape[0], int)
    for b in np.nonzero(leaf)[0]:
        lo, hi = t["isrcse"][b]
        cnt[t["isrc"][lo:hi + 1]] += 1
    assert np.all(cnt == 1)
    # colleague relation symmetric and 2:1 balance of touching leaves
    for b in range(nb):
        for j in t["nbors"][b, :t["nnbors"][b]]:
            assert b in t["nbors"][j, :t["nnbors"][j]]
    lev = t["ilevel"]
    cen = t["centers"]
    bs = t["boxsize"]
    lb = np.nonzero(leaf)[0]
    for i in lb[::7]:
        d = np.max(np.abs(cen[lb] - cen[i]) - ((bs[lev[lb]] + bs[lev[i]]) / 2)[:, None], axis=1)
        touch = lb[d <= 1e-12]
        assert np.all(np.abs(lev[touch] - lev[i]) <= 1)


def _golden_files():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz")) if os.path.isdir(GOLDEN) else []


@pytest.mark.parametrize("fname", _golden_files())
def test_golden_fixtures(oracle, fname):
    """The oracle reproduces its committed fixtures (tests/golden/make_golden.py)."""
    d = np.load(os.path.join(GOLDEN, fname), allow_pickle=False)
    kw = dict(charge=d["charge"], ifpgh=int(d["ifpgh"]), bs0=float(d["bs0"]),
              cen0=list(d["cen0"]))
    if d["targets"].shape[0]:
        kw["targets"] = d["targets"]
        kw["ifpghtarg"] = int(d["ifpghtarg"])
    r = oracle.pfgt(int(d["nd"]), int(d["dim"]), float(d["delta"]), float(d["eps"]),
                    int(d["iperiod"]), d["sources"], **kw)
    for f in ("pot", "grad", "pottarg", "gradtarg"):
        if f in d.files and f in r:
            np.testing.assert_allclose(r[f], d[f], rtol=1e-12, atol=1e-14)


def _cdh_reference_hessian(dim, delta, src, q, rn, ds, trg):
    """The Hessian of gnd_directcdh as the reference writes it
    (src/pfgt/pfgt_direct.f:510-598, one density, no cut-off): the dipole
    terms use dg = (-2/delta)(t - s) in the gnd_directdh formula."""
    nh = dim * (dim + 1) // 2
    pairs = [(k, k) for k in range(dim)] + [(k, j) for k in range(dim) for j in range(k + 1, dim)]
    if dim == 2:
        pairs = [(0, 0), (0, 1), (1, 1)]
    rfac = -2.0 / delta
    out = np.zeros((trg.shape[0], nh))
    for t in range(trg.shape[0]):
        dr = trg[t] - src
        e = np.exp(-np.sum(dr * dr, axis=1) / delta)
        dg = rfac * dr
        rinc = -np.sum(dg * rn, axis=1)
        rincg = -rn * rfac + rinc[:, None] * dg
        for m, (k, j) in enumerate(pairs):
            ch = (rfac if k == j else 0.0) + dg[:, k] * dg[:, j]
            if k == j:
                dh = -rfac * (dg[:, k] * rn[:, k] + rinc) - rincg[:, k] * dg[:, k]
            else:
                dh = -rfac * dg[:, k] * rn[:, j] - rincg[:, k] * dg[:, j]
            out[t, m] = np.sum(e * (ch * q[:, 0] + dh * ds[:, 0]))
    return out


@pytest.mark.parametrize("dim", [2, 3])
def test_combined_charge_dipole_hessian_is_the_true_hessian(oracle, dim):
    """Charges and dipoles with hessians: the oracle (and the GPU library)
    return the Hessian of the potential, checked here against central
    differences of the gradient.  The reference's gnd_directcdh formula
    differs from it (flipped rinc/rincg terms); the restatement of that
    formula above must fail the same check, which documents the departure."""
    rng = np.random.default_rng(31 + dim)
    ns, nt, delta = 40, 6, 0.05
    src = rng.uniform(-0.2, 0.2, (ns, dim))
    q = rng.uniform(-1, 1, (ns, 1))
    ds = rng.uniform(-1, 1, (ns, 1))
    rn = rng.standard_normal((ns, dim))
    trg = rng.uniform(-0.15, 0.15, (nt, dim))
    kw = dict(charge=q, dipstr=ds, rnormal=rn)
    r = oracle.direct_exact(1, dim, delta, src, trg, ifpgh=3, **kw)
    h = 1e-5
    pairs = [(k, k) for k in range(dim)] + [(k, j) for k in range(dim) for j in range(k + 1, dim)]
    if dim == 2:
        pairs = [(0, 0), (0, 1), (1, 1)]
    fd = np.zeros((nt, len(pairs)))
    for m, (k, j) in enumerate(pairs):
        tp, tm = trg.copy(), trg.copy()
        tp[:, j] += h
        tm[:, j] -= h
        gp = oracle.direct_exact(1, dim, delta, src, tp, ifpgh=2, **kw)["grad"][:, k, 0]
        gm = oracle.direct_exact(1, dim, delta, src, tm, ifpgh=2, **kw)["grad"][:, k, 0]
        fd[:, m] = (gp - gm) / (2 * h)
    assert relerr(fd, r["hess"][:, :, 0]) < 1e-6
    ref_cdh = _cdh_reference_hessian(dim, delta, src, q, rn, ds, trg)
    assert relerr(fd, ref_cdh) > 1e-2
