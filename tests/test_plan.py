"""Reusable plans (fgt_plan_create/execute/destroy): executing a plan with
some strengths must give the results of a single pfgt call with the same
points and strengths; the plan's geometry is reused across executions."""
import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu, relerr
from fgt_b200 import workloads as W


def _tol(eps):
    return 1e-6 if eps >= 1e-6 else 1e-12  # mixed path: FP32 sums in another order


def test_plan_argument_errors(fgt):
    L = fgt.lib()
    L.fgt_plan_create.restype = C.c_void_p
    L.fgt_plan_execute.restype = C.c_int
    st = C.c_int(-1)
    b0 = C.c_double(1.0)
    c0 = np.zeros(3)
    h = L.fgt_plan_create(None, 1, 4, C.c_double(1e-3), C.c_double(1e-6), 0, C.byref(b0),
                          c0.ctypes.data_as(C.c_void_p), 10, None, 0, None, C.byref(st))
    assert not h and st.value == fgt.FGT_ERR_ARG
    assert L.fgt_plan_execute(None, 1, None, 0, None, None, 1, None, None, None, 0, None, None,
                              None) == fgt.FGT_ERR_ARG
    L.fgt_plan_destroy(None)  # no-op


@pytest.mark.skipif(has_gpu(), reason="checks the no-device status")
def test_plan_without_device(fgt):
    src = np.random.default_rng(0).uniform(-0.5, 0.5, (100, 3))
    with pytest.raises(fgt.FgtError) as e:
        fgt.Plan(1, 3, 1e-3, 1e-6, 0, src)
    assert e.value.code == fgt.FGT_ERR_NODEVICE


CASES = [
    ("3d_sphere_grad_targets", dict(nd=1, dim=3, delta=1e-3, eps=1e-6, iperiod=0), 30000, 4000, 2,
     False),
    ("3d_fp64_eps1e-9", dict(nd=1, dim=3, delta=3e-4, eps=1e-9, iperiod=0), 8000, 0, 2, False),
    ("2d_periodic_nd2", dict(nd=2, dim=2, delta=1e-4, eps=1e-6, iperiod=1, bs0=1.0,
                             cen0=[0.0, 0.0]), 20000, 2000, 2, False),
    ("2d_dipole_hess", dict(nd=1, dim=2, delta=1e-3, eps=1e-6, iperiod=0), 5000, 0, 3, True),
]


def _oracle_tol(eps):
    return 0.3 * eps if eps < 1e-6 else 1e-6  # FP64 path below 1e-6, mixed at and above


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_plan_matches_single_calls(fgt, oracle, case):
    name, geo, ns, nt, pgh, dip = case
    rng = np.random.default_rng(5)
    dim, nd = geo["dim"], geo["nd"]
    src = W.sphere_surface(rng, ns, radius=0.35) if dim == 3 else W.uniform(rng, ns, dim)
    trg = W.uniform(rng, nt, dim) if nt else None
    plan = fgt.Plan(sources=src, targets=trg, **geo)
    try:
        for rep in range(3):  # several executions with new strengths
            kw = dict(charge=rng.uniform(-1, 1, (ns, nd)), ifpgh=pgh,
                      ifpghtarg=pgh if nt else 0)
            if dip:
                kw.update(dipstr=rng.uniform(-1, 1, (ns, nd)), rnormal=rng.standard_normal((ns, dim)))
            r = plan.execute(**kw)
            one = fgt.pfgt(sources=src, targets=trg, **geo, **kw)
            if rep == 0:  # the plan against the restated reference
                ro = oracle.pfgt(sources=src, targets=trg, **geo, **kw)
                for f in ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg"):
                    if f in ro:
                        e = relerr(ro[f], r[f])
                        assert e < _oracle_tol(geo["eps"]), (name, f, e)
            for f in ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg"):
                if f in one:
                    assert relerr(one[f], r[f]) < _tol(geo["eps"]), (name, rep, f,
                                                                     relerr(one[f], r[f]))
        assert plan.bs0 == one["bs0"]
    finally:
        plan.close()
