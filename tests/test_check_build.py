"""The FGT_CHECK build, libfgt_b200_check.so: every kernel's indexed
accesses are bounds-checked on the device; a failed check records a site
number, skips the access (no trap) and the call returns FGT_ERR_CHECK.  It is
the stand-in for a memory checker (none can run on the GPUs used here).

CPU: the checked library loads and exports the header's symbols; the normal
library reports that it has no checks.  GPU: a host-crafted out-of-range
index trips a check (and the library stays usable), and the checked build
gives the normal build's results on the parity cases without tripping."""
import os

import numpy as np
import pytest

from conftest import relerr
from fgt_b200 import workloads as W


@pytest.fixture(scope="module")
def checked(fgt):
    if not os.path.exists(fgt.LIB_CHECK_PATH):
        from fgt_b200 import build as b
        b.build(check=True)
    return fgt.lib(check=True)


def test_checked_library_exports_header_symbols(fgt, checked):
    from test_abi import header_functions
    for n in header_functions():
        assert hasattr(checked, n), n


def test_normal_build_has_no_checks(fgt):
    assert fgt.lib().fgt_check_selftest() == fgt.FGT_ERR_UNSUPPORTED
    assert "without FGT_CHECK" in fgt.last_error()


@pytest.mark.gpu
def test_crafted_index_trips_a_check(fgt, checked):
    assert checked.fgt_check_selftest() == fgt.FGT_ERR_CHECK
    assert "site 103" in fgt.last_error(check=True)
    # the check word is cleared: the next call runs clean
    rng = np.random.default_rng(2)
    src = W.uniform(rng, 3000, 2)
    r = fgt.pfgt(1, 2, 1e-3, 1e-6, 0, src, charge=rng.uniform(-1, 1, (3000, 1)), ifpgh=2,
                 check=True)
    assert np.isfinite(r["pot"]).all()


def _cases():
    rng = np.random.default_rng(23)
    u = W.uniform
    c5 = W.config(5, scale=0.004, delta=1e-3, eps=1e-6)
    c5 = {k: v for k, v in c5.items() if k != "name"}
    return [
        ("3d_sphere_pw_direct", c5),
        ("3d_root_split", {k: v for k, v in W.config(5, scale=0.02, delta=1e-1).items()
                           if k != "name"}),
        ("2d_periodic_nd2_small_boxes", dict(nd=2, dim=2, delta=1e-3, eps=1e-6, iperiod=1,
                                             bs0=1.0, cen0=[0.0, 0.0], sources=u(rng, 20000, 2),
                                             charge=rng.uniform(-1, 1, (20000, 2)), ifpgh=2)),
        ("2d_dipole_hess", dict(nd=1, dim=2, delta=1e-3, eps=1e-6, iperiod=0,
                                sources=u(rng, 5000, 2), charge=rng.uniform(-1, 1, (5000, 1)),
                                dipstr=rng.uniform(-1, 1, (5000, 1)),
                                rnormal=rng.standard_normal((5000, 2)), ifpgh=3)),
        ("3d_eps1e-9_targets", dict(nd=1, dim=3, delta=1e-3, eps=1e-9, iperiod=0,
                                    sources=W.gaussian_clusters(rng, 6000, 3, ncl=4),
                                    charge=rng.uniform(-1, 1, (6000, 1)), ifpgh=2,
                                    targets=u(rng, 500, 3), ifpghtarg=2)),
    ]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", _cases(), ids=[c[0] for c in _cases()])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_checked_build_matches_normal_build(fgt, checked, name, kw, prec):
    p = fgt.PREC_MIXED if prec == "mixed" else fgt.PREC_FP64
    a = fgt.pfgt(precision=p, **kw)
    b = fgt.pfgt(precision=p, check=True, **kw)  # raises FgtError on a failed check
    # FP32 shared-memory atomics of the spreading add in a run-dependent
    # order: the mixed path agrees to FP32 rounding, the FP64 path closely
    tol = 1e-6 if prec == "mixed" else 1e-12
    for f in ("pot", "grad", "hess", "pottarg", "gradtarg", "hesstarg"):
        if f in a:
            assert relerr(a[f], b[f]) < tol, (name, prec, f, relerr(a[f], b[f]))
