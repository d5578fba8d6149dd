"""The FP32 near field has two kernels: the packed list-1 source stream
(charges, one density, potential or potential + gradient) and the list
walk (every other case, and the packed case above its record cap).  Both
must give the same sums; FGT_NEAR_PACK_MAX=0 forces the walk."""
import numpy as np
import pytest

from conftest import relerr
from fgt_b200 import workloads as W


def _cases():
    rng = np.random.default_rng(5)
    cfg = W.config(5, scale=0.004, delta=1e-3, eps=1e-6)  # sphere + background, PW + direct
    kw = {k: v for k, v in cfg.items() if k != "name"}
    yield "headline_reduced", kw
    n = 3000
    yield "direct_only_2d", dict(nd=1, dim=2, delta=1e-2, eps=1e-6, iperiod=0,
                                 sources=W.uniform(rng, n, 2), charge=rng.uniform(-1, 1, (n, 1)),
                                 ifpgh=2, targets=W.uniform(rng, 700, 2), ifpghtarg=1)
    yield "periodic_3d", dict(nd=1, dim=3, delta=2e-3, eps=1e-6, iperiod=1, bs0=1.0,
                              cen0=[0.0, 0.0, 0.0], sources=W.uniform(rng, 6000, 3),
                              charge=rng.uniform(-1, 1, (6000, 1)), ifpgh=2)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", list(_cases()), ids=[c[0] for c in _cases()])
def test_packed_and_walking_near_field_agree(fgt, monkeypatch, name, kw):
    packed = fgt.pfgt(precision=fgt.PREC_MIXED, stats=True, **kw)
    if name != "periodic_3d":
        assert packed["stats"]["near_pairs"] > 0, name
    monkeypatch.setenv("FGT_NEAR_PACK_MAX", "0")
    walked = fgt.pfgt(precision=fgt.PREC_MIXED, **kw)
    monkeypatch.delenv("FGT_NEAR_PACK_MAX")
    ref = fgt.pfgt(precision=fgt.PREC_FP64, **kw)
    for f in ("pot", "grad", "pottarg", "gradtarg"):
        if f in packed:
            # FP32 pair sums grouped differently: agreement at the FP32 level
            assert relerr(walked[f], packed[f]) < 1e-6, (name, f)
            # the mixed path against the FP64 path at eps = 1e-6
            assert relerr(ref[f], packed[f]) < 2e-6, (name, f)
