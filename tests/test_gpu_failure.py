"""Failure detection on the GPU without a fault: the packed near-field
kernel's waits on its bulk copies are bounded (0.2 s).  With
FGT_TEST_NEAR_STALL=1 the kernel omits its first copy, so that wait runs out;
the kernel records FGT_ERR_TIMEOUT, lets its other copy land and returns, and
the call reports the status.  The context stays usable: the next call gives
the normal result."""
import numpy as np
import pytest

from conftest import relerr
from fgt_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_near_field_wait_timeout_is_reported(fgt, monkeypatch):
    cfg = W.config(5, scale=0.002, delta=1e-3, eps=1e-6)
    kw = {k: v for k, v in cfg.items() if k != "name"}
    ref = fgt.pfgt(precision=fgt.PREC_MIXED, stats=True, **kw)
    assert ref["stats"]["near_pairs"] > 0
    monkeypatch.setenv("FGT_TEST_NEAR_STALL", "1")
    with pytest.raises(fgt.FgtError) as e:
        fgt.pfgt(precision=fgt.PREC_MIXED, **kw)
    assert e.value.code == fgt.FGT_ERR_TIMEOUT
    assert "ran out" in fgt.last_error()
    monkeypatch.delenv("FGT_TEST_NEAR_STALL")
    again = fgt.pfgt(precision=fgt.PREC_MIXED, **kw)
    for f in ("pot", "grad", "pottarg", "gradtarg"):
        assert relerr(ref[f], again[f]) < 1e-6, f
