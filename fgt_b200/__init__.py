"""fgt_b200 -- B200-native discrete point fast Gauss transform.

Python mirror of the reference Fortran entry point
``pfgt(nd,dim,delta,eps,iperiod,bs0,cen0,ns,sources,ifcharge,charge,
ifdipole,rnormal,dipstr,ifpgh,pot,grad,hess,nt,targ,ifpghtarg,pottarg,
gradtarg,hesstarg)`` (src/pfgt/pfgt.f:6-10) over the C ABI of
include/fgt_b200.h (libfgt_b200.so, CUDA sm_100a).  There is no CPU
fallback: without the built library or a CUDA device every call raises.

numpy layouts (C order) equal the reference's column-major layouts:
sources (ns, dim), charge (ns, nd), pot (n, nd), grad (n, dim, nd),
hess (n, nhess, nd).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfgt_b200.so")
LIB_CHECK_PATH = os.path.join(_HERE, "libfgt_b200_check.so")  # FGT_CHECK build

FGT_OK = 0
FGT_ERR_ARG = 1
FGT_ERR_CUDA = 2
FGT_ERR_NOMEM = 3
FGT_ERR_UNSUPPORTED = 4
FGT_ERR_TIMEOUT = 5
FGT_ERR_NODEVICE = 6
FGT_ERR_INJECTED = 7
FGT_ERR_CHECK = 8

PREC_AUTO = 0
PREC_FP64 = 1
PREC_MIXED = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class FgtStats(C.Structure):
    _fields_ = [
        ("nlevels", C.c_int), ("nboxes", C.c_int), ("npwlevel", C.c_int), ("npw", C.c_int),
        ("ndiv", C.c_int), ("precision_used", C.c_int), ("n_form_boxes", C.c_int),
        ("n_eval_boxes", C.c_int), ("n_eval_nufft", C.c_int), ("n_translations", C.c_int),
        ("spread_width", C.c_int), ("grid_cells", C.c_int), ("n_kernel_launches", C.c_int),
        ("near_pairs", C.c_double), ("flops_form", C.c_double), ("flops_eval", C.c_double),
        ("flops_direct", C.c_double), ("bytes_translate", C.c_double),
        ("pts_form", C.c_double), ("pts_eval_nufft", C.c_double),
        ("pts_eval_modal", C.c_double), ("bs0", C.c_double), ("cen0", C.c_double * 3),
        ("ms", C.c_double * 12), ("small_eval_used", C.c_int), ("tuned", C.c_int),
        ("slabs_form", C.c_int), ("slabs_eval", C.c_int),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("cen0", "ms")}
        d["cen0"] = list(self.cen0)
        d["ms"] = list(self.ms)
        return d


class FgtOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int), ("device_ptrs", C.c_int), ("device", C.c_int),
        ("stream", C.c_void_p), ("ndiv", C.c_int), ("small_eval", C.c_int),
        ("spread_width", C.c_int), ("timing", C.c_int), ("stats", C.POINTER(FgtStats)),
        ("root_level", C.c_int), ("autotune", C.c_int),
    ]


class FgtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fgt_b200 error {code}: {msg}")
        self.code = code


_lib = None

# every symbol declared in include/fgt_b200.h
class FgtInstance(C.Structure):
    """Mirror of `fgt_instance` (include/fgt_b200.h)."""
    _fields_ = [("nd", C.c_int), ("dim", C.c_int), ("delta", C.c_double), ("eps", C.c_double),
                ("iperiod", C.c_int), ("bs0", C.c_void_p), ("cen0", C.c_void_p),
                ("ns", C.c_int), ("sources", C.c_void_p), ("ifcharge", C.c_int),
                ("charge", C.c_void_p), ("ifdipole", C.c_int), ("rnormal", C.c_void_p),
                ("dipstr", C.c_void_p), ("ifpgh", C.c_int), ("pot", C.c_void_p),
                ("grad", C.c_void_p), ("hess", C.c_void_p), ("nt", C.c_int),
                ("targ", C.c_void_p), ("ifpghtarg", C.c_int), ("pottarg", C.c_void_p),
                ("gradtarg", C.c_void_p), ("hesstarg", C.c_void_p), ("status", C.c_int)]


EXPORTS = ["fgt_opts_default", "fgt_pfgt_c", "pfgt_", "pfgt_direct_", "fgt_last_status",
           "fgt_last_error", "fgt_version", "fgt_debug_tree_build", "fgt_debug_tree_get",
           "fgt_debug_tree_free", "fgt_direct_nomalloc", "fgt_pfgt_batch", "fgt_plan_create",
           "fgt_plan_execute", "fgt_plan_destroy", "fgt_check_selftest"]


_libs = {}


def lib(check=False):
    """Load libfgt_b200.so, or with check=True the FGT_CHECK build
    libfgt_b200_check.so (raises if it is missing: no CPU fallback)."""
    global _lib
    if check:
        if "check" not in _libs:
            _libs["check"] = _load(LIB_CHECK_PATH, "python -m fgt_b200.build --check")
        return _libs["check"]
    if _lib is None:
        _lib = _load(LIB_PATH, "python -m fgt_b200.build")
    return _lib


def _load(path, how):
    if True:
        if not os.path.exists(path):
            raise FgtError(FGT_ERR_NODEVICE, f"{path} not built; run {how}")
        L = C.CDLL(path)
        L.fgt_pfgt_c.restype = C.c_int
        L.fgt_pfgt_c.argtypes = [
            C.POINTER(FgtOpts), C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _dp, _dp,
            C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
            C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
            C.c_void_p, C.c_void_p, C.c_void_p]
        L.fgt_last_error.restype = C.c_char_p
        L.fgt_version.restype = C.c_char_p
        L.fgt_debug_tree_build.restype = C.c_void_p
        L.fgt_debug_tree_build.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                           _dp, C.c_int, _dp, C.c_int, _dp, C.c_int]
        L.fgt_debug_tree_get.restype = C.c_long
        L.fgt_debug_tree_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_long]
        L.fgt_debug_tree_free.argtypes = [C.c_void_p]
        L.fgt_check_selftest.restype = C.c_int
        L.fgt_check_selftest.argtypes = []
    return L


def version():
    return lib().fgt_version().decode()


def last_error(check=False):
    return lib(check).fgt_last_error().decode()


def _f64(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def pfgt(nd, dim, delta, eps, iperiod, sources, charge=None, dipstr=None, rnormal=None,
         ifpgh=1, targets=None, ifpghtarg=0, bs0=1.0, cen0=None, precision=PREC_AUTO,
         ndiv=0, small_eval=-1, spread_width=0, stats=False, timing=False, check=False,
         root_level=-1, autotune=0):
    """Point FGT with the reference's argument meaning (src/pfgt/pfgt.f:11-53).

    Returns a dict with pot/grad/hess (sources) and pottarg/gradtarg/hesstarg
    (targets) for the requested levels, plus bs0/cen0 (and stats if asked).
    check=True runs the FGT_CHECK build (device bounds checks).
    root_level >= 0 (free space): bs0/cen0 are inputs and root_level is the
    cut-off level (a spatial shard of a larger point set).
    autotune: 1 use tuned parameters from the cache, 2 also tune on a miss.
    """
    L = lib(check)
    src = _f64(sources, (-1, dim))
    ns = src.shape[0]
    trg = None if targets is None else _f64(targets, (-1, dim))
    nt = 0 if trg is None else trg.shape[0]
    nhess = dim * (dim + 1) // 2
    ifcharge = 0 if charge is None else 1
    ifdipole = 0 if dipstr is None else 1
    q = _f64(charge, (ns, nd)) if ifcharge else None
    ds = _f64(dipstr, (ns, nd)) if ifdipole else None
    rn = _f64(rnormal, (ns, dim)) if ifdipole else None
    pot = np.zeros((ns, nd)) if ifpgh >= 1 else None
    grad = np.zeros((ns, dim, nd)) if ifpgh >= 2 else None
    hess = np.zeros((ns, nhess, nd)) if ifpgh >= 3 else None
    pt = np.zeros((nt, nd)) if (ifpghtarg >= 1 and nt) else None
    gt = np.zeros((nt, dim, nd)) if (ifpghtarg >= 2 and nt) else None
    ht = np.zeros((nt, nhess, nd)) if (ifpghtarg >= 3 and nt) else None
    b0 = C.c_double(float(bs0))
    c0 = np.zeros(3)
    if cen0 is not None:
        c0[:dim] = np.asarray(cen0, dtype=np.float64)[:dim]
    st = FgtStats()
    o = FgtOpts()
    L.fgt_opts_default(C.byref(o))
    o.precision = precision
    o.ndiv = ndiv
    o.small_eval = small_eval
    o.spread_width = spread_width
    o.timing = 1 if timing else 0
    o.stats = C.pointer(st) if (stats or timing) else None
    o.root_level = root_level
    o.autotune = autotune
    rc = L.fgt_pfgt_c(C.byref(o), nd, dim, delta, eps, iperiod, C.byref(b0),
                      c0.ctypes.data_as(_dp), ns, _ptr(src), ifcharge, _ptr(q), ifdipole,
                      _ptr(rn), _ptr(ds), ifpgh, _ptr(pot), _ptr(grad), _ptr(hess), nt,
                      _ptr(trg), ifpghtarg if nt else 0, _ptr(pt), _ptr(gt), _ptr(ht))
    if rc != FGT_OK:
        raise FgtError(rc, last_error(check))
    out = {"bs0": b0.value, "cen0": c0[:dim].copy()}
    for k, v in (("pot", pot), ("grad", grad), ("hess", hess), ("pottarg", pt),
                 ("gradtarg", gt), ("hesstarg", ht)):
        if v is not None:
            out[k] = v
    if stats or timing:
        out["stats"] = st.as_dict()
    return out


def pfgt_batch(instances, precision=PREC_AUTO, nworkers=0, ndiv=0, small_eval=-1, autotune=0):
    """Many independent point FGTs in one call (host arrays).

    `instances` is a list of dicts with the keyword arguments of `pfgt`
    (nd, dim, delta, eps, iperiod, sources, charge, dipstr, rnormal, ifpgh,
    targets, ifpghtarg, bs0, cen0).  Returns one result dict per instance, as
    `pfgt` does; raises FgtError if any instance failed.
    """
    L = lib()
    keep, outs = [], []
    arr = (FgtInstance * len(instances))()
    for x, (kw) in zip(arr, instances):
        nd, dim = kw["nd"], kw["dim"]
        src = _f64(kw["sources"], (-1, dim))
        ns = src.shape[0]
        trg = kw.get("targets")
        trg = None if trg is None else _f64(trg, (-1, dim))
        nt = 0 if trg is None else trg.shape[0]
        ifpgh, ifpghtarg = kw.get("ifpgh", 1), kw.get("ifpghtarg", 0) if nt else 0
        nhess = dim * (dim + 1) // 2
        q = _f64(kw["charge"], (ns, nd)) if kw.get("charge") is not None else None
        ds = _f64(kw["dipstr"], (ns, nd)) if kw.get("dipstr") is not None else None
        rn = _f64(kw["rnormal"], (ns, dim)) if ds is not None else None
        o = {"pot": np.zeros((ns, nd)) if ifpgh >= 1 else None,
             "grad": np.zeros((ns, dim, nd)) if ifpgh >= 2 else None,
             "hess": np.zeros((ns, nhess, nd)) if ifpgh >= 3 else None,
             "pottarg": np.zeros((nt, nd)) if ifpghtarg >= 1 else None,
             "gradtarg": np.zeros((nt, dim, nd)) if ifpghtarg >= 2 else None,
             "hesstarg": np.zeros((nt, nhess, nd)) if ifpghtarg >= 3 else None}
        b0 = np.array([float(kw.get("bs0", 1.0))])
        c0 = np.zeros(3)
        if kw.get("cen0") is not None:
            c0[:dim] = np.asarray(kw["cen0"], dtype=np.float64)[:dim]
        keep += [src, trg, q, ds, rn, b0, c0]
        x.nd, x.dim, x.delta, x.eps = nd, dim, kw["delta"], kw["eps"]
        x.iperiod = kw.get("iperiod", 0)
        x.bs0, x.cen0 = _ptr(b0), _ptr(c0)
        x.ns, x.sources = ns, _ptr(src)
        x.ifcharge, x.charge = (1 if q is not None else 0), _ptr(q)
        x.ifdipole, x.rnormal, x.dipstr = (1 if ds is not None else 0), _ptr(rn), _ptr(ds)
        x.ifpgh, x.pot, x.grad, x.hess = ifpgh, _ptr(o["pot"]), _ptr(o["grad"]), _ptr(o["hess"])
        x.nt, x.targ, x.ifpghtarg = nt, _ptr(trg), ifpghtarg
        x.pottarg, x.gradtarg, x.hesstarg = _ptr(o["pottarg"]), _ptr(o["gradtarg"]), _ptr(o["hesstarg"])
        outs.append((o, b0, c0, dim))
    opts = FgtOpts()
    L.fgt_opts_default(C.byref(opts))
    opts.precision = precision
    opts.ndiv = ndiv
    opts.small_eval = small_eval
    opts.autotune = autotune
    L.fgt_pfgt_batch.restype = C.c_int
    rc = L.fgt_pfgt_batch(C.byref(opts), len(instances), arr, nworkers)
    if rc != FGT_OK:
        bad = [i for i, x in enumerate(arr) if x.status != FGT_OK]
        raise FgtError(rc, f"instances {bad[:8]} failed")
    res = []
    for o, b0, c0, dim in outs:
        r = {k: v for k, v in o.items() if v is not None}
        r["bs0"], r["cen0"] = float(b0[0]), c0[:dim].copy()
        res.append(r)
    return res


class Plan:
    """Reusable plan (fgt_plan_create/execute/destroy): the tree, lists and
    sorted point offsets of fixed sources and targets kept on the device for
    repeated evaluations with new strengths (host arrays)."""

    def __init__(self, nd, dim, delta, eps, iperiod, sources, targets=None, bs0=1.0, cen0=None,
                 precision=PREC_AUTO, ndiv=0, small_eval=-1):
        L = lib()
        L.fgt_plan_create.restype = C.c_void_p
        L.fgt_plan_execute.restype = C.c_int
        self.nd, self.dim = nd, dim
        self._src = _f64(sources, (-1, dim))
        self.ns = self._src.shape[0]
        self._trg = None if targets is None else _f64(targets, (-1, dim))
        self.nt = 0 if self._trg is None else self._trg.shape[0]
        b0 = C.c_double(float(bs0))
        c0 = np.zeros(3)
        if cen0 is not None:
            c0[:dim] = np.asarray(cen0, dtype=np.float64)[:dim]
        o = FgtOpts()
        L.fgt_opts_default(C.byref(o))
        o.precision, o.ndiv, o.small_eval = precision, ndiv, small_eval
        st = C.c_int(0)
        self._h = L.fgt_plan_create(C.byref(o), nd, dim, C.c_double(delta), C.c_double(eps),
                                    iperiod, C.byref(b0),
                                    c0.ctypes.data_as(_dp), self.ns, _ptr(self._src), self.nt,
                                    _ptr(self._trg), C.byref(st))
        if not self._h:
            raise FgtError(st.value, last_error())
        self.bs0, self.cen0 = b0.value, c0[:dim].copy()

    def execute(self, charge=None, dipstr=None, rnormal=None, ifpgh=1, ifpghtarg=0):
        """Results of pfgt on the plan's points for these strengths (dict as `pfgt`)."""
        L = lib()
        nd, dim, ns, nt = self.nd, self.dim, self.ns, self.nt
        nhess = dim * (dim + 1) // 2
        q = _f64(charge, (ns, nd)) if charge is not None else None
        ds = _f64(dipstr, (ns, nd)) if dipstr is not None else None
        rn = _f64(rnormal, (ns, dim)) if ds is not None else None
        ifpghtarg = ifpghtarg if nt else 0
        out = {"pot": np.zeros((ns, nd)) if ifpgh >= 1 else None,
               "grad": np.zeros((ns, dim, nd)) if ifpgh >= 2 else None,
               "hess": np.zeros((ns, nhess, nd)) if ifpgh >= 3 else None,
               "pottarg": np.zeros((nt, nd)) if ifpghtarg >= 1 else None,
               "gradtarg": np.zeros((nt, dim, nd)) if ifpghtarg >= 2 else None,
               "hesstarg": np.zeros((nt, nhess, nd)) if ifpghtarg >= 3 else None}
        rc = L.fgt_plan_execute(C.c_void_p(self._h), 1 if q is not None else 0, _ptr(q),
                                1 if ds is not None else 0, _ptr(rn), _ptr(ds), ifpgh,
                                _ptr(out["pot"]), _ptr(out["grad"]), _ptr(out["hess"]), ifpghtarg,
                                _ptr(out["pottarg"]), _ptr(out["gradtarg"]), _ptr(out["hesstarg"]))
        if rc != FGT_OK:
            raise FgtError(rc, last_error())
        return {k: v for k, v in out.items() if v is not None}

    def close(self):
        if getattr(self, "_h", None):
            lib().fgt_plan_destroy(C.c_void_p(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pfgt_device(opts, nd, dim, delta, eps, iperiod, bs0, cen0, ns, src_ptr, ifcharge,
                q_ptr, ifdipole, rn_ptr, ds_ptr, ifpgh, pot_ptr, grad_ptr, hess_ptr, nt,
                trg_ptr, ifpghtarg, pt_ptr, gt_ptr, ht_ptr):
    """Raw call with device pointers (opts.device_ptrs must be 1)."""
    L = lib()
    b0 = C.c_double(float(bs0))
    c0 = np.zeros(3)
    c0[:dim] = np.asarray(cen0, dtype=np.float64)[:dim]
    rc = L.fgt_pfgt_c(C.byref(opts), nd, dim, delta, eps, iperiod, C.byref(b0),
                      c0.ctypes.data_as(_dp), ns, src_ptr, ifcharge, q_ptr, ifdipole, rn_ptr,
                      ds_ptr, ifpgh, pot_ptr, grad_ptr, hess_ptr, nt, trg_ptr, ifpghtarg,
                      pt_ptr, gt_ptr, ht_ptr)
    if rc != FGT_OK:
        raise FgtError(rc, last_error())
    return b0.value, c0[:dim].copy()


_TREE_ARRAYS = {
    "key": np.uint64, "level": np.int32, "nonleaf": np.int32, "parent": np.int32,
    "child0": np.int32, "center": np.float64, "src_lo": np.int32, "src_hi": np.int32,
    "trg_lo": np.int32, "trg_hi": np.int32, "isrc": np.uint32, "itrg": np.uint32,
    "l1_ptr": np.int32, "l1_src": np.int32, "form_box": np.int32, "eval_box": np.int32,
    "eval_self": np.int32, "trans_ptr": np.int32, "trans_src": np.int32, "trans_w": np.int32,
    "scalars": np.int32, "dscalars": np.float64,
}


def debug_tree(dim, delta, eps, iperiod, sources, targets, bs0=1.0, cen0=None, ndiv=0):
    """Device-built tree and lists of a pfgt call, copied to numpy arrays."""
    L = lib()
    src = _f64(sources, (-1, dim))
    trg = _f64(targets, (-1, dim)) if targets is not None and len(targets) else np.zeros((0, dim))
    c0 = np.zeros(3)
    if cen0 is not None:
        c0[:dim] = np.asarray(cen0, dtype=np.float64)[:dim]
    h = L.fgt_debug_tree_build(dim, delta, eps, iperiod, float(bs0), c0.ctypes.data_as(_dp),
                               src.shape[0], src.ctypes.data_as(_dp), trg.shape[0],
                               trg.ctypes.data_as(_dp) if trg.shape[0] else None, ndiv)
    if not h:
        raise FgtError(FGT_ERR_NODEVICE, "debug tree build failed: " + last_error())
    out = {}
    try:
        for name, dt in _TREE_ARRAYS.items():
            n = L.fgt_debug_tree_get(h, name.encode(), None, 0)
            a = np.zeros(max(n, 0), dtype=dt)
            if n > 0:
                L.fgt_debug_tree_get(h, name.encode(), a.ctypes.data_as(C.c_void_p), n)
            out[name] = a
    finally:
        L.fgt_debug_tree_free(h)
    sc = out.pop("scalars")
    (out["nlevels"], out["nboxes"], out["npwlevel"], out["ncutoff"], out["nleaves"],
     out["n_form"], out["n_eval"], out["n_trans"], out["n_l1"], out["D"], out["nlevend"],
     out["iperiod0"]) = [int(v) for v in sc]
    ds = out.pop("dscalars")
    out["bs0"] = float(ds[0])
    out["cen0"] = ds[1:1 + dim].copy()
    out["boxsize"] = ds[4:].copy()
    out["center"] = out["center"].reshape(-1, dim)
    return out
