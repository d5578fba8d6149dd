"""fgt_direct_nomalloc: the allocation-free variant of the all-pairs direct
sum (static device scratch, caller-owned device buffers), checked against
the existing pfgt_direct_ entry point through the C ABI.

Collected last (file name) so that it also runs after every other test in
one process; it passes alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import relerr

TOL = 1e-12  # both paths are FP64 all-pairs sums; only the summation order differs


def _proto(L):
    f = L.fgt_direct_nomalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                  C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                  C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fgt_last_error.restype = C.c_char_p
    return f


def test_nomalloc_rejects_outputs_beyond_scratch(fgt):
    """Size check happens before any device work: runs without a GPU."""
    L = fgt.lib()
    f = _proto(L)
    nt = (8 << 20) // 8 // 4 + 1  # 3D pot+grad: 4 doubles per target, one target too many
    rc = f(1, 3, 1e-3, 1.0, None, 10, None, 1, None, 0, None, None, nt, None, 2, None, None,
           None, None)
    assert rc == fgt.FGT_ERR_UNSUPPORTED
    assert b"static scratch" in L.fgt_last_error()


def _reference(L, nd, dim, delta, dmax, shift, src, q, rn, ds, trg, pgh):
    """The existing entry point: pfgt_direct_ on host arrays (gfortran ABI)."""
    nt, nh = trg.shape[0], dim * (dim + 1) // 2
    pot = np.zeros((nt, nd))
    grad = np.zeros((nt, dim, nd))
    hess = np.zeros((nt, nh, nd))
    i = lambda v: C.byref(C.c_int(v))
    d = lambda v: C.byref(C.c_double(v))
    p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    L.pfgt_direct_(i(nd), i(dim), d(delta), d(dmax), i(1 if shift is not None else 0),
                   p(shift if shift is not None else np.zeros(dim)), i(1), i(src.shape[0]), i(1),
                   i(nt), p(src), i(1 if q is not None else 0), p(q), i(1 if ds is not None else 0),
                   p(rn), p(ds), p(trg), i(pgh), p(pot), p(grad), p(hess))
    assert L.fgt_last_status() == 0
    return pot, grad, hess


@pytest.mark.gpu
def test_nomalloc_matches_pfgt_direct_on_two_calls(fgt):
    import torch
    L = fgt.lib()
    f = _proto(L)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    # A call with no targets computes nothing; it only loads the module and
    # resolves the scratch address (the warm-up a pool-owning host makes).
    rc = f(1, 3, 1e-3, 1.0, None, 10, None, 1, None, 0, None, None, 0, None, 1, None, None,
           None, C.c_void_p(stream.cuda_stream))
    assert rc == 0, L.fgt_last_error()
    # Calls in a row with different shapes: each has another target count,
    # dimension, density count or field set than the one before, so stale
    # accumulators of an earlier call would show.
    calls = [
        dict(nd=1, dim=3, ns=7000, nt=2500, pgh=3, charge=True, dipole=True, shift=None,
             delta=2e-3, dmax=2e-3 * np.log(1e16)),
        dict(nd=1, dim=2, ns=3000, nt=400, pgh=2, charge=True, dipole=False,
             shift=np.array([1.0, 0.0]), delta=5e-2, dmax=1e30),
        dict(nd=2, dim=1, ns=2000, nt=900, pgh=1, charge=False, dipole=True, shift=None,
             delta=1e-3, dmax=1e-3 * np.log(1e12)),
        dict(nd=3, dim=3, ns=4000, nt=700, pgh=3, charge=True, dipole=False, shift=None,
             delta=1e-2, dmax=1e30),
    ]
    for c in calls:
        nd, dim, ns, nt, pgh = c["nd"], c["dim"], c["ns"], c["nt"], c["pgh"]
        nh = dim * (dim + 1) // 2
        src = rng.uniform(-0.5, 0.5, (ns, dim))
        trg = rng.uniform(-0.5, 0.5, (nt, dim))
        if c["shift"] is not None:
            trg[:, 0] += 1.0  # targets near the shifted image of the sources
        q = rng.uniform(-1, 1, (ns, nd)) if c["charge"] else None
        rn = rng.standard_normal((ns, dim)) if c["dipole"] else None
        ds = rng.uniform(-1, 1, (ns, nd)) if c["dipole"] else None
        ref = _reference(L, nd, dim, c["delta"], c["dmax"], c["shift"], src, q, rn, ds, trg,
                         pgh)

        t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        dsrc, dtrg, dq, drn, dds = t(src), t(trg), t(q), t(rn), t(ds)
        pot = torch.zeros((nt, nd), dtype=torch.float64, device=dev)
        grad = torch.zeros((nt, dim, nd), dtype=torch.float64, device=dev)
        hess = torch.zeros((nt, nh, nd), dtype=torch.float64, device=dev)
        ptr = lambda a: None if a is None else a.data_ptr()
        sh = c["shift"]
        torch.cuda.synchronize()
        rc = f(nd, dim, c["delta"], c["dmax"],
               None if sh is None else sh.ctypes.data_as(C.c_void_p), ns, ptr(dsrc),
               1 if q is not None else 0, ptr(dq), 1 if ds is not None else 0, ptr(drn), ptr(dds),
               nt, ptr(dtrg), pgh, ptr(pot), ptr(grad) if pgh >= 2 else None,
               ptr(hess) if pgh >= 3 else None, C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.fgt_last_error()
        torch.cuda.synchronize()
        got = (pot.cpu().numpy(), grad.cpu().numpy(), hess.cpu().numpy())
        for name, k in (("pot", 0), ("grad", 1), ("hess", 2)):
            if k + 1 > pgh:
                continue
            assert np.abs(ref[k]).max() > 0
            assert relerr(ref[k], got[k]) < TOL, (name, nd, dim, relerr(ref[k], got[k]))
