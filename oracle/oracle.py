"""ctypes front end of the CPU restatement in pfgt_oracle.c.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, never by the product package.

Array conventions follow the reference's column-major layouts seen from numpy
in C order: sources (ns, dim), charge (ns, nd), pot (n, nd), grad
(n, dim, nd), hess (n, nhess, nd).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle_pfgt.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _TreeT(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nlevels", C.c_int), ("nboxes", C.c_int),
        ("npwlevel", C.c_int), ("ndiv", C.c_int),
        ("bs0", C.c_double), ("cen0", C.c_double * 3),
        ("ilevel", _ip), ("iparent", _ip), ("nchild", _ip), ("nnbors", _ip),
        ("nbors", _ip), ("laddr", _ip),
        ("centers", _dp), ("boxsize", _dp),
        ("isrc", _ip), ("isrcse", _ip), ("itrg", _ip), ("itrgse", _ip),
        ("ifpwexp", _ip), ("nlistpw", _ip), ("listpw", _ip), ("nlist1", _ip),
        ("list1", _ip),
        ("mnbors", C.c_int), ("mlistpw", C.c_int), ("mlist1", C.c_int),
        ("npw", C.c_int), ("pmax", C.c_double),
    ]


def build():
    """Compile the restatement (make -C oracle)."""
    src = os.path.join(_HERE, "pfgt_oracle.c")
    if (not os.path.exists(_LIB)) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
        _lib.oracle_tree_build.restype = C.POINTER(_TreeT)
        _lib.oracle_tree_build.argtypes = [
            C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, _dp, C.c_int, _dp,
            C.c_int, _dp, C.c_int]
        _lib.oracle_tree_free.argtypes = [C.POINTER(_TreeT)]
        _lib.oracle_pfgt.restype = C.c_int
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def tree(dim, delta, eps, iperiod, sources, targets, bs0=1.0, cen0=None, ndiv=0):
    """Tree, sorted permutations and lists of pfgt (0-based box ids)."""
    L = lib()
    src = _f64(sources).reshape(-1, dim)
    trg = _f64(targets).reshape(-1, dim)
    c0 = np.zeros(3) if cen0 is None else _f64(list(cen0) + [0.0] * (3 - dim))
    r = L.oracle_tree_build(dim, delta, eps, iperiod, float(bs0), _p(c0), src.shape[0],
                            _p(src), trg.shape[0], _p(trg), int(ndiv))
    t = r.contents
    nb, nl = t.nboxes, t.nlevels

    def ia(ptr, n):
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n > 0 else np.zeros(0, np.int32)

    def da(ptr, n):
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n > 0 else np.zeros(0)

    out = dict(
        dim=dim, nlevels=nl, nboxes=nb, npwlevel=t.npwlevel, ndiv=t.ndiv, bs0=t.bs0,
        cen0=np.array(t.cen0[:dim]), npw=t.npw, pmax=t.pmax,
        ilevel=ia(t.ilevel, nb), iparent=ia(t.iparent, nb), nchild=ia(t.nchild, nb),
        nnbors=ia(t.nnbors, nb), nbors=ia(t.nbors, nb * t.mnbors).reshape(nb, t.mnbors),
        laddr=ia(t.laddr, 2 * (nl + 1)).reshape(nl + 1, 2),
        centers=da(t.centers, nb * dim).reshape(nb, dim), boxsize=da(t.boxsize, nl + 1),
        isrc=ia(t.isrc, src.shape[0]), isrcse=ia(t.isrcse, 2 * nb).reshape(nb, 2),
        itrg=ia(t.itrg, trg.shape[0]), itrgse=ia(t.itrgse, 2 * nb).reshape(nb, 2),
        ifpwexp=ia(t.ifpwexp, nb), nlistpw=ia(t.nlistpw, nb),
        listpw=ia(t.listpw, nb * max(t.mlistpw, 1)).reshape(nb, max(t.mlistpw, 1)),
        nlist1=ia(t.nlist1, nb), list1=ia(t.list1, nb * t.mlist1).reshape(nb, t.mlist1),
    )
    L.oracle_tree_free(r)
    return out


def pfgt(nd, dim, delta, eps, iperiod, sources, charge=None, dipstr=None,
         rnormal=None, ifpgh=1, targets=None, ifpghtarg=0, bs0=1.0, cen0=None,
         quirks=0, nufft="exact", root_level=None):
    """Restated reference pfgt; returns dict(pot, grad, hess, pottarg, ...).

    root_level (free space, not None): bs0/cen0 are inputs and the cut-off
    level is root_level, the geometry of a larger point set this one is a
    shard of.
    nufft="exact": plane-wave sums by exact non-uniform DFTs (the checker);
    nufft="spread": the restatement's own ES-kernel NUFFT, OpenMP over boxes
    (the timed CPU baseline).  quirks: bit 0/1/2 reproduce the reference's
    ifpgh==ifpghtarg skip, nd>1 scramble and empty small-root result.
    """
    L = lib()
    src = _f64(sources).reshape(-1, dim)
    ns = src.shape[0]
    trg = np.zeros((0, dim)) if targets is None else _f64(targets).reshape(-1, dim)
    nt = trg.shape[0]
    nhess = dim * (dim + 1) // 2
    ifcharge = 0 if charge is None else 1
    ifdipole = 0 if dipstr is None else 1
    q = _f64(charge).reshape(ns, nd) if ifcharge else np.zeros(1)
    ds = _f64(dipstr).reshape(ns, nd) if ifdipole else np.zeros(1)
    rn = _f64(rnormal).reshape(ns, dim) if ifdipole else np.zeros(1)
    pot = np.zeros((max(ns, 1), nd))
    grad = np.zeros((max(ns, 1), dim, nd))
    hess = np.zeros((max(ns, 1), nhess, nd))
    pt = np.zeros((max(nt, 1), nd))
    gt = np.zeros((max(nt, 1), dim, nd))
    ht = np.zeros((max(nt, 1), nhess, nd))
    b0 = C.c_double(float(bs0))
    c0 = np.zeros(3) if cen0 is None else _f64(list(cen0) + [0.0] * (3 - dim))
    L.oracle_set_root_level(C.c_int(-1 if root_level is None else int(root_level)))
    L.oracle_pfgt(C.c_int(nd), C.c_int(dim), C.c_double(delta), C.c_double(eps),
                  C.c_int(iperiod), C.byref(b0), _p(c0), C.c_int(ns), _p(src),
                  C.c_int(ifcharge), _p(q), C.c_int(ifdipole), _p(rn), _p(ds),
                  C.c_int(ifpgh), _p(pot), _p(grad), _p(hess), C.c_int(nt),
                  _p(trg if nt else np.zeros(1)), C.c_int(ifpghtarg), _p(pt), _p(gt),
                  _p(ht), C.c_int(quirks), C.c_int(1 if nufft == "spread" else 0))
    L.oracle_set_root_level(C.c_int(-1))
    out = dict(bs0=b0.value, cen0=c0[:dim].copy())
    if ifpgh >= 1:
        out["pot"] = pot[:ns]
    if ifpgh >= 2:
        out["grad"] = grad[:ns]
    if ifpgh >= 3:
        out["hess"] = hess[:ns]
    if ifpghtarg >= 1:
        out["pottarg"] = pt[:nt]
    if ifpghtarg >= 2:
        out["gradtarg"] = gt[:nt]
    if ifpghtarg >= 3:
        out["hesstarg"] = ht[:nt]
    return out


def threads():
    """OpenMP threads the restatement uses."""
    return int(lib().oracle_threads())


def direct_exact(nd, dim, delta, sources, evalpts, charge=None, dipstr=None,
                 rnormal=None, ifpgh=1, iperiod=0, bs0=1.0, nimg=None):
    """Exact FP64 Gauss transform at evalpts (no truncation, self included).

    Periodic: images |n_d| <= nimg with nimg defaulting to
    ceil(sqrt(delta*ln(1e16))/bs0) + 1.
    """
    L = lib()
    src = _f64(sources).reshape(-1, dim)
    ns = src.shape[0]
    tg = _f64(evalpts).reshape(-1, dim)
    nt = tg.shape[0]
    nhess = dim * (dim + 1) // 2
    if nimg is None:
        nimg = int(np.ceil(np.sqrt(delta * np.log(1e16)) / bs0)) + 1 if iperiod else 0
    ifcharge = 0 if charge is None else 1
    ifdipole = 0 if dipstr is None else 1
    q = _f64(charge).reshape(ns, nd) if ifcharge else np.zeros(1)
    ds = _f64(dipstr).reshape(ns, nd) if ifdipole else np.zeros(1)
    rn = _f64(rnormal).reshape(ns, dim) if ifdipole else np.zeros(1)
    pot = np.zeros((nt, nd))
    grad = np.zeros((nt, dim, nd))
    hess = np.zeros((nt, nhess, nd))
    L.oracle_direct_exact(C.c_int(nd), C.c_int(dim), C.c_double(delta), C.c_int(iperiod),
                          C.c_double(bs0), C.c_int(nimg), C.c_int(ns), _p(src),
                          C.c_int(ifcharge), _p(q), C.c_int(ifdipole), _p(rn), _p(ds),
                          C.c_int(nt), _p(tg), C.c_int(ifpgh), _p(pot), _p(grad), _p(hess))
    out = {"pot": pot}
    if ifpgh >= 2:
        out["grad"] = grad
    if ifpgh >= 3:
        out["hess"] = hess
    return out


def relerr(ref, approx):
    """Relative l2 error of the reference test's `derr`
    (test/pfgt/test_pfgt_all.f:496-512)."""
    ref = np.asarray(ref).ravel()
    approx = np.asarray(approx).ravel()
    n = np.linalg.norm(ref)
    return float(np.linalg.norm(ref - approx) / (n if n > 0 else 1.0))
