"""GPU pfgt parity through the C ABI against the oracle (the restatement of
the reference, exact plane-wave sums) and the exact FP64 Gauss transform.

Tolerances (relative l2 per field, the reference's `derr`):
  FP64 path vs oracle:   0.3*eps (the path's own NUFFT is the only change)
  mixed path vs oracle:  eps (FP32 bulk arithmetic, FP64 geometry/accumulation)
  either path vs exact:  the oracle's own error plus the above.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import relerr
from fgt_b200 import workloads as W

pytestmark = pytest.mark.gpu

FIELDS = ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg")


def _case_list():
    rng = np.random.default_rng(7)
    u = W.uniform
    return [
        ("3d_direct", dict(nd=1, dim=3, delta=1e-4, eps=1e-6, iperiod=0, sources=u(rng, 20000, 3),
                           charge=rng.uniform(-1, 1, (20000, 1)), ifpgh=1)),
        ("3d_pw_eps1e-3", dict(nd=1, dim=3, delta=1e-2, eps=1e-3, iperiod=0,
                               sources=u(rng, 20000, 3), charge=rng.uniform(-1, 1, (20000, 1)),
                               ifpgh=2)),
        ("3d_pw_eps1e-6", dict(nd=1, dim=3, delta=3e-3, eps=1e-6, iperiod=0,
                               sources=W.gaussian_clusters(rng, 8000, 3, ncl=4),
                               charge=rng.standard_normal((8000, 1)), ifpgh=2,
                               targets=u(rng, 1000, 3), ifpghtarg=1)),
        ("2d_pw_targets", dict(nd=1, dim=2, delta=1e-4, eps=1e-6, iperiod=0,
                               sources=W.gaussian_clusters(rng, 20000, 2, ncl=8),
                               charge=rng.uniform(-1, 1, (20000, 1)), ifpgh=2,
                               targets=u(rng, 3000, 2), ifpghtarg=2)),
        ("2d_periodic_nd2", dict(nd=2, dim=2, delta=1e-4, eps=1e-6, iperiod=1, bs0=1.0,
                                 cen0=[0.0, 0.0], sources=u(rng, 20000, 2),
                                 charge=rng.uniform(-1, 1, (20000, 2)), ifpgh=2)),
        ("2d_periodic_small_level", dict(nd=1, dim=2, delta=3e-2, eps=1e-6, iperiod=1, bs0=1.0,
                                         cen0=[0.0, 0.0], sources=u(rng, 3000, 2),
                                         charge=rng.uniform(-1, 1, (3000, 1)), ifpgh=2)),
        ("2d_dipole_hess", dict(nd=1, dim=2, delta=1e-3, eps=1e-6, iperiod=0,
                                sources=u(rng, 5000, 2), charge=rng.uniform(-1, 1, (5000, 1)),
                                dipstr=rng.uniform(-1, 1, (5000, 1)),
                                rnormal=rng.standard_normal((5000, 2)), ifpgh=3)),
        ("3d_dipole_only", dict(nd=1, dim=3, delta=1e-2, eps=1e-3, iperiod=0,
                                sources=u(rng, 6000, 3), dipstr=rng.uniform(-1, 1, (6000, 1)),
                                rnormal=rng.standard_normal((6000, 3)), ifpgh=3)),
        ("1d_hess_eps1e-9", dict(nd=1, dim=1, delta=1e-4, eps=1e-9, iperiod=0,
                                 sources=u(rng, 3000, 1), charge=rng.uniform(-1, 1, (3000, 1)),
                                 ifpgh=3, targets=u(rng, 500, 1), ifpghtarg=3)),
        ("3d_root_pw", dict(nd=1, dim=3, delta=1.0, eps=1e-6, iperiod=0, sources=u(rng, 2000, 3),
                            charge=rng.uniform(-1, 1, (2000, 1)), ifpgh=2)),
        ("2d_small_root_direct", dict(nd=1, dim=2, delta=1.0, eps=1e-6, iperiod=0,
                                      sources=u(rng, 50, 2) * 0.01,
                                      charge=rng.uniform(-1, 1, (50, 1)), ifpgh=2)),
    ] + _benchmark_regime_cases()


def _benchmark_regime_cases():
    """Reduced-size cases in the regimes of the benchmark configurations:
    3D at eps = 1e-9 and 1e-12 (npw 40 and 54; the FP64 grids exceed shared
    memory, so form and evaluation run on global-memory grids), the
    clustered sources with separate targets of configuration 2, the 2D
    periodic multi-density field of configuration 3, 3D periodic (free-space
    and periodic plane-wave nodes), several densities in 3D, and the
    sphere + background point set at delta = 1e-1 (cut-off level 0: one
    root box holds every point)."""
    rng = np.random.default_rng(17)
    u = W.uniform
    c5 = W.config(5, scale=0.0005, delta=1e-1, eps=1e-6)
    c5 = {k: v for k, v in c5.items() if k != "name"}
    c5e3 = W.config(5, scale=0.002, delta=1e-1, eps=1e-3)
    c5e3 = {k: v for k, v in c5e3.items() if k != "name"}
    return [
        ("3d_eps1e-9", dict(nd=1, dim=3, delta=1e-3, eps=1e-9, iperiod=0,
                            sources=W.gaussian_clusters(rng, 6000, 3, ncl=4),
                            charge=rng.uniform(-1, 1, (6000, 1)), ifpgh=2,
                            targets=u(rng, 500, 3), ifpghtarg=2)),
        ("3d_eps1e-12", dict(nd=1, dim=3, delta=1e-3, eps=1e-12, iperiod=0,
                             sources=W.gaussian_clusters(rng, 2500, 3, ncl=3),
                             charge=rng.uniform(-1, 1, (2500, 1)), ifpgh=2,
                             targets=u(rng, 300, 3), ifpghtarg=1)),
        ("config2_clusters_eps1e-9", dict(nd=1, dim=3, delta=1e-5, eps=1e-9, iperiod=0,
                                          sources=W.gaussian_clusters(rng, 10000, 3, ncl=8),
                                          charge=rng.standard_normal((10000, 1)), ifpgh=2,
                                          targets=u(rng, 10000, 3), ifpghtarg=2)),
        ("config3_periodic_nd4", dict(nd=4, dim=2, delta=1e-3, eps=1e-6, iperiod=1, bs0=1.0,
                                      cen0=[0.0, 0.0], sources=u(rng, 20000, 2),
                                      charge=rng.uniform(-1, 1, (20000, 4)), ifpgh=2)),
        ("3d_periodic_pw", dict(nd=1, dim=3, delta=4e-3, eps=1e-6, iperiod=1, bs0=1.0,
                                cen0=[0.0, 0.0, 0.0], sources=u(rng, 20000, 3),
                                charge=rng.uniform(-1, 1, (20000, 1)), ifpgh=2)),
        ("3d_periodic_nodes", dict(nd=1, dim=3, delta=1e-2, eps=1e-6, iperiod=1, bs0=1.0,
                                   cen0=[0.0, 0.0, 0.0], sources=u(rng, 20000, 3),
                                   charge=rng.uniform(-1, 1, (20000, 1)), ifpgh=2)),
        ("3d_nd3", dict(nd=3, dim=3, delta=3e-3, eps=1e-6, iperiod=0,
                        sources=W.gaussian_clusters(rng, 4000, 3, ncl=4),
                        charge=rng.uniform(-1, 1, (4000, 3)), ifpgh=2,
                        targets=u(rng, 400, 3), ifpghtarg=1)),
        ("config5_delta1e-1_root", c5),
        ("config5_delta1e-1_eps1e-3", c5e3),
        # drawn last: the cases above keep the points of the shared generator
        ("3d_hess_dipole_eps1e-9", dict(nd=1, dim=3, delta=1e-3, eps=1e-9, iperiod=0,
                                        sources=W.gaussian_clusters(rng, 3000, 3, ncl=3),
                                        charge=rng.uniform(-1, 1, (3000, 1)),
                                        dipstr=rng.uniform(-1, 1, (3000, 1)),
                                        rnormal=rng.standard_normal((3000, 3)), ifpgh=3,
                                        targets=u(rng, 300, 3), ifpghtarg=3)),
    ]


CASES = _case_list()
SLAB_CASES = ("3d_eps1e-9", "3d_hess_dipole_eps1e-9", "3d_eps1e-12", "config2_clusters_eps1e-9")
_ORACLE = {}


def oracle_result(oracle, name, kw):
    """The oracle's output of a named case, computed once per session."""
    if name not in _ORACLE:
        _ORACLE[name] = oracle.pfgt(**kw)
    return _ORACLE[name]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pfgt_matches_oracle(fgt, oracle, case, prec):
    name, kw = case
    p = fgt.PREC_FP64 if prec == "fp64" else fgt.PREC_MIXED
    r = fgt.pfgt(precision=p, stats=True, **kw)
    ro = oracle_result(oracle, name, kw)
    if name in ("3d_eps1e-9", "3d_hess_dipole_eps1e-9", "3d_eps1e-12",
                "config2_clusters_eps1e-9", "3d_periodic_pw", "3d_periodic_nodes", "3d_nd3",
                "config3_periodic_nd4",
                "config5_delta1e-1_root", "config5_delta1e-1_eps1e-3"):
        assert r["stats"]["n_form_boxes"] > 0, (name, r["stats"])  # the plane-wave path ran
    if name in SLAB_CASES:
        # 3D grids beyond shared memory: evaluated in x-slabs; formed in
        # x-slabs in FP32 (FP64 forms keep a global-memory grid)
        assert r["stats"]["slabs_eval"] > 1, (name, r["stats"])
        assert (r["stats"]["slabs_form"] > 1) == (prec == "mixed"), (name, r["stats"])
    # mixed: FP32 bulk arithmetic resolves about 1e-6 (below eps = 1e-6,
    # outside the precision policy, the W^3 = 1728-2744 cell stencils of the
    # eps = 1e-9 / 1e-12 kernels land at 1-2e-6 on some point sets)
    if prec == "fp64":
        tol = 0.3 * kw["eps"]
    else:
        tol = max(0.3 * kw["eps"], 1e-6 if kw["eps"] >= 1e-6 else 3e-6)
    for f in FIELDS:
        if f in ro:
            assert f in r
            e = relerr(ro[f], r[f])
            assert e <= tol, (name, prec, f, e, tol)
    assert r["stats"]["precision_used"] == p
    np.testing.assert_allclose(r["bs0"], ro["bs0"], rtol=0, atol=0)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_config1_full_size_vs_exact(fgt, oracle, prec):
    """Benchmark configuration 1 at full size (N = 1e5, uniform, delta 1e-4,
    eps 1e-6, potential): the whole answer is the direct near field."""
    cfg = W.config(1)
    kw = {k: v for k, v in cfg.items() if k != "name"}
    p = fgt.PREC_FP64 if prec == "fp64" else fgt.PREC_MIXED
    r = fgt.pfgt(precision=p, **kw)
    rng = np.random.default_rng(W.SEED0 + 2)
    idx = rng.choice(kw["sources"].shape[0], 1000, replace=False)
    ex = oracle.direct_exact(1, 3, kw["delta"], kw["sources"], kw["sources"][idx],
                             charge=kw["charge"], ifpgh=1)
    ro = oracle.pfgt(**kw)
    assert relerr(ex["pot"], r["pot"][idx]) < 2e-6
    assert relerr(ro["pot"], r["pot"]) < (1e-12 if prec == "fp64" else 1e-6)


def test_headline_distribution_reduced(fgt, oracle):
    """Sphere + background distribution of the headline at N = M = 4e4 with
    delta chosen so the plane-wave path and the direct path both run."""
    cfg = W.config(5, scale=0.004, delta=1e-3, eps=1e-6)
    kw = {k: v for k, v in cfg.items() if k != "name"}
    r64 = fgt.pfgt(precision=fgt.PREC_FP64, stats=True, **kw)
    r32 = fgt.pfgt(precision=fgt.PREC_MIXED, stats=True, **kw)
    assert r32["stats"]["n_form_boxes"] > 0 and r32["stats"]["near_pairs"] > 0
    rng = np.random.default_rng(1)
    idx = rng.choice(kw["sources"].shape[0], 500, replace=False)
    ex = oracle.direct_exact(1, 3, kw["delta"], kw["sources"], kw["sources"][idx],
                             charge=kw["charge"], ifpgh=2)
    for r in (r64, r32):
        assert relerr(ex["pot"], r["pot"][idx]) < 2e-6
        assert relerr(ex["grad"], r["grad"][idx]) < 1e-5
        assert relerr(r["pot"], r["pottarg"]) < 1e-12  # targets are the same points
    assert relerr(r64["pot"], r32["pot"]) < 1e-6


def test_single_source_gaussian_on_gpu(fgt):
    s = np.array([[0.1, -0.2, 0.05]])
    rng = np.random.default_rng(0)
    t = s + rng.uniform(-0.05, 0.05, (300, 3))
    delta, eps = 1e-3, 1e-6
    r = fgt.pfgt(1, 3, delta, eps, 0, s, charge=np.ones((1, 1)), ifpgh=1, targets=t,
                 ifpghtarg=2, precision=fgt.PREC_FP64)
    rr = np.sum((t - s) ** 2, axis=1)
    ex = np.where(rr < delta * np.log(1 / eps), np.exp(-rr / delta), 0.0)
    np.testing.assert_allclose(r["pottarg"][:, 0], ex, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(r["pot"][0, 0], 1.0)


def test_periodic_face_pairs_on_gpu(fgt):
    rng = np.random.default_rng(5)
    n = 20000
    src = rng.uniform(0, 1, (n, 2))
    q = rng.uniform(0, 1, (n, 1))
    nx = 12
    h = 1.0 / (nx + 1)
    lo = [[i * h, 0.0] for i in range(1, nx + 1)] + [[0.0, i * h] for i in range(1, nx + 1)]
    hi = [[p[0], 1.0] if p[1] == 0.0 else [1.0, p[1]] for p in lo]
    trg = np.array(lo + hi)
    for prec in (fgt.PREC_FP64, fgt.PREC_MIXED):
        r = fgt.pfgt(1, 2, 1e-4, 1e-6, 1, src, charge=q, ifpgh=1, targets=trg, ifpghtarg=2,
                     bs0=1.0, cen0=[0.5, 0.5], precision=prec)
        half = len(lo)
        assert relerr(r["pottarg"][:half], r["pottarg"][half:]) < 2e-6


def test_device_pointer_path_matches_host_path(fgt):
    import torch
    cfg = W.config(5, scale=0.002, delta=1e-3, eps=1e-6)
    kw = {k: v for k, v in cfg.items() if k != "name"}
    r = fgt.pfgt(precision=fgt.PREC_MIXED, **kw)
    dev = torch.device("cuda", 0)
    N = kw["sources"].shape[0]
    s = torch.from_numpy(kw["sources"]).to(dev)
    t = torch.from_numpy(kw["targets"]).to(dev)
    q = torch.from_numpy(kw["charge"]).to(dev)
    pot = torch.empty((N, 1), dtype=torch.float64, device=dev)
    grad = torch.empty((N, 3, 1), dtype=torch.float64, device=dev)
    pt = torch.empty((N, 1), dtype=torch.float64, device=dev)
    gt = torch.empty((N, 3, 1), dtype=torch.float64, device=dev)
    o = fgt.FgtOpts()
    fgt.lib().fgt_opts_default(C.byref(o))
    o.precision = fgt.PREC_MIXED
    o.device_ptrs = 1
    o.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    fgt.pfgt_device(o, 1, 3, kw["delta"], kw["eps"], 0, 1.0, [0, 0, 0], N, s.data_ptr(), 1,
                    q.data_ptr(), 0, None, None, 2, pot.data_ptr(), grad.data_ptr(), None, N,
                    t.data_ptr(), 2, pt.data_ptr(), gt.data_ptr(), None)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(pot.cpu().numpy(), r["pot"])
    np.testing.assert_array_equal(gt.cpu().numpy(), r["gradtarg"])


def test_fortran_dropins(fgt, oracle):
    """pfgt_ and pfgt_direct_ with by-reference arguments (gfortran ABI)."""
    L = fgt.lib()
    rng = np.random.default_rng(3)
    n, nt = 4000, 300
    src = rng.uniform(-0.5, 0.5, (n, 3))
    q = rng.uniform(-1, 1, (n, 1))
    trg = rng.uniform(-0.5, 0.5, (nt, 3))
    pot = np.zeros((n, 1))
    pt = np.zeros((nt, 1))
    gt = np.zeros((nt, 3, 1))
    i = lambda v: C.byref(C.c_int(v))
    d = lambda v: C.byref(C.c_double(v))
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    b0 = C.c_double(0.0)
    c0 = np.zeros(3)
    L.pfgt_(i(1), i(3), d(1e-3), d(1e-6), i(0), C.byref(b0), p(c0), i(n), p(src), i(1), p(q),
            i(0), None, None, i(1), p(pot), None, None, i(nt), p(trg), i(2), p(pt), p(gt), None)
    assert L.fgt_last_status() == 0
    ro = oracle.pfgt(1, 3, 1e-3, 1e-6, 0, src, charge=q, ifpgh=1, targets=trg, ifpghtarg=2)
    assert relerr(ro["pot"], pot) < 1e-6
    assert relerr(ro["gradtarg"], gt) < 1e-6
    assert b0.value == ro["bs0"]
    # pfgt_direct_: all pairs, FP64, incremented outputs
    dp = np.zeros((nt, 1))
    dg = np.zeros((nt, 3, 1))
    sh = np.zeros(3)
    L.pfgt_direct_(i(1), i(3), d(1e-3), d(1e30), i(0), p(sh), i(1), i(n), i(1), i(nt), p(src),
                   i(1), p(q), i(0), None, None, p(trg), i(2), p(dp), p(dg), None)
    ex = oracle.direct_exact(1, 3, 1e-3, src, trg, charge=q, ifpgh=2)
    np.testing.assert_allclose(dp, ex["pot"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(dg, ex["grad"], rtol=1e-11, atol=1e-10)
