"""fgt_pfgt_batch: many independent point FGTs in one call must give each
instance the results of a single fgt_pfgt_c call with the same options."""
import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu, relerr
from fgt_b200 import workloads as W


def test_batch_argument_errors(fgt):
    L = fgt.lib()
    L.fgt_pfgt_batch.restype = C.c_int
    assert L.fgt_pfgt_batch(None, -1, None, 0) == fgt.FGT_ERR_ARG
    assert L.fgt_pfgt_batch(None, 3, None, 0) == fgt.FGT_ERR_ARG
    assert L.fgt_pfgt_batch(None, 0, None, 0) == fgt.FGT_OK


@pytest.mark.skipif(has_gpu(), reason="checks the no-device status")
def test_batch_without_device_reports_every_instance(fgt):
    L = fgt.lib()
    L.fgt_pfgt_batch.restype = C.c_int
    arr = (fgt.FgtInstance * 3)()
    for x in arr:
        x.status = 12345
    assert L.fgt_pfgt_batch(None, 3, arr, 2) == fgt.FGT_ERR_NODEVICE
    assert all(x.status == fgt.FGT_ERR_NODEVICE for x in arr)


def _instances():
    rng = np.random.default_rng(21)
    u = W.uniform
    out = []
    for i in range(14):  # 3D charge, pot only, sizes and parameters of the batched workload
        n = int(np.exp(rng.uniform(np.log(500), np.log(20000))))
        src = u(rng, n, 3) if i % 2 else W.sphere_surface(rng, n, radius=0.35)
        out.append(dict(nd=1, dim=3, delta=float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-2)))),
                        eps=float(rng.choice([1e-3, 1e-6])), iperiod=0, sources=src,
                        charge=rng.uniform(-1, 1, (n, 1)), ifpgh=1))
    out.append(dict(nd=2, dim=2, delta=1e-4, eps=1e-6, iperiod=0, sources=u(rng, 6000, 2),
                    charge=rng.uniform(-1, 1, (6000, 2)), ifpgh=2, targets=u(rng, 900, 2),
                    ifpghtarg=2))
    out.append(dict(nd=1, dim=2, delta=1e-3, eps=1e-6, iperiod=1, bs0=1.0, cen0=[0.0, 0.0],
                    sources=u(rng, 4000, 2), charge=rng.uniform(-1, 1, (4000, 1)), ifpgh=2))
    out.append(dict(nd=1, dim=3, delta=3e-3, eps=1e-6, iperiod=0, sources=u(rng, 5000, 3),
                    charge=rng.uniform(-1, 1, (5000, 1)), dipstr=rng.uniform(-1, 1, (5000, 1)),
                    rnormal=rng.standard_normal((5000, 3)), ifpgh=3))
    out.append(dict(nd=1, dim=1, delta=1e-4, eps=1e-9, iperiod=0, sources=u(rng, 3000, 1),
                    charge=rng.uniform(-1, 1, (3000, 1)), ifpgh=3, targets=u(rng, 400, 1),
                    ifpghtarg=3))
    return out


def _tol(kw):
    return 1e-6 if kw["eps"] >= 1e-6 else 1e-12  # mixed: FP32 sums in another order


@pytest.mark.gpu
def test_batch_matches_single_calls(fgt):
    inst = _instances()
    res = fgt.pfgt_batch(inst, nworkers=6)
    assert len(res) == len(inst)
    for kw, r in zip(inst, res):
        one = fgt.pfgt(**kw)
        for f in ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg"):
            if f in one:
                assert f in r
                assert relerr(one[f], r[f]) < _tol(kw), (f, kw["dim"], kw["eps"], relerr(one[f], r[f]))
        assert r["bs0"] == one["bs0"]


@pytest.mark.gpu
def test_batch_bad_instance_does_not_stop_the_others(fgt):
    L = fgt.lib()
    inst = _instances()[:6]
    ref = [fgt.pfgt(**kw) for kw in inst]
    # a direct C call so that one instance can be made invalid (ns = 0)
    arr = (fgt.FgtInstance * len(inst))()
    keep = []
    for x, kw in zip(arr, inst):
        src = np.ascontiguousarray(kw["sources"])
        q = np.ascontiguousarray(kw["charge"])
        pot = np.zeros((src.shape[0], 1))
        b0, c0 = np.array([1.0]), np.zeros(3)
        keep.append((src, q, pot, b0, c0))
        x.nd, x.dim, x.delta, x.eps, x.iperiod = 1, 3, kw["delta"], kw["eps"], 0
        x.bs0, x.cen0 = fgt._ptr(b0), fgt._ptr(c0)
        x.ns, x.sources, x.ifcharge, x.charge = src.shape[0], fgt._ptr(src), 1, fgt._ptr(q)
        x.ifpgh, x.pot = 1, fgt._ptr(pot)
    arr[2].ns = 0
    L.fgt_pfgt_batch.restype = C.c_int
    rc = L.fgt_pfgt_batch(None, len(inst), arr, 4)
    assert rc == fgt.FGT_ERR_ARG
    for i, (x, k) in enumerate(zip(arr, keep)):
        if i == 2:
            assert x.status == fgt.FGT_ERR_ARG
        else:
            assert x.status == fgt.FGT_OK
            assert relerr(ref[i]["pot"], k[2]) < _tol(inst[i])
