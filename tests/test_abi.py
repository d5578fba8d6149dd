"""CPU tests of the C ABI: the library loads, exports every symbol declared
in include/fgt_b200.h, validates arguments and reports host-side failures
(fault injection) without touching a GPU."""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "fgt_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = re.sub(r"^\s*#.*$", "", txt, flags=re.M)  # preprocessor lines are not declarations
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", txt)))


def test_library_exports_header_symbols(fgt):
    L = fgt.lib()
    names = header_functions()
    assert "fgt_pfgt_c" in names and "pfgt_" in names and "pfgt_direct_" in names
    for n in names:
        assert hasattr(L, n), n
    assert set(fgt.EXPORTS) <= set(names)
    assert fgt.version().startswith("fgt_b200")


def _call(fgt, **over):
    L = fgt.lib()
    n, dim, nd = 10, 2, 1
    src = np.random.default_rng(0).uniform(-0.5, 0.5, (n, dim))
    q = np.ones((n, nd))
    pot = np.zeros((n, nd))
    args = dict(nd=nd, dim=dim, delta=1e-3, eps=1e-6, iperiod=0)
    args.update(over)
    b0 = C.c_double(1.0)
    c0 = np.zeros(3)
    o = fgt.FgtOpts()
    L.fgt_opts_default(C.byref(o))
    rc = L.fgt_pfgt_c(C.byref(o), args["nd"], args["dim"], args["delta"], args["eps"],
                      args["iperiod"], C.byref(b0), c0.ctypes.data_as(C.POINTER(C.c_double)),
                      n, src.ctypes.data_as(C.c_void_p), 1, q.ctypes.data_as(C.c_void_p), 0,
                      None, None, 1, pot.ctypes.data_as(C.c_void_p), None, None, 0, None, 0,
                      None, None, None)
    return rc


@pytest.mark.parametrize("over", [dict(dim=4), dict(nd=0), dict(eps=0.0), dict(eps=2.0),
                                  dict(delta=-1.0), dict(iperiod=3)])
def test_argument_errors(fgt, over):
    assert _call(fgt, **over) == fgt.FGT_ERR_ARG
    assert fgt.last_error()


def _run_child(code, env):
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       cwd=ROOT, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_fault_injection_status_and_nan_fill():
    """FGT_FAULT makes the host path fail before any device work: the status
    call returns FGT_ERR_INJECTED and the Fortran drop-in NaN-fills its
    requested outputs and records the status."""
    code = r"""
import ctypes as C, numpy as np, fgt_b200 as F
L = F.lib()
n = 8
src = np.random.default_rng(0).uniform(size=(n, 3))
q = np.ones((n, 1)); pot = np.zeros((n, 1)); grad = np.zeros((n, 3, 1))
try:
    F.pfgt(1, 3, 1e-3, 1e-6, 0, src, charge=q, ifpgh=1)
    raise SystemExit("no error")
except F.FgtError as e:
    assert e.code == F.FGT_ERR_INJECTED, e.code
i = lambda v: C.byref(C.c_int(v)); d = lambda v: C.byref(C.c_double(v))
b0 = C.c_double(1.0); c0 = np.zeros(3)
L.pfgt_(i(1), i(3), d(1e-3), d(1e-6), i(0), C.byref(b0), c0.ctypes.data_as(C.c_void_p), i(n),
        src.ctypes.data_as(C.c_void_p), i(1), q.ctypes.data_as(C.c_void_p), i(0), None, None,
        i(2), pot.ctypes.data_as(C.c_void_p), grad.ctypes.data_as(C.c_void_p), None, i(0), None,
        i(0), None, None, None)
assert L.fgt_last_status() == F.FGT_ERR_INJECTED
assert np.all(np.isnan(pot)) and np.all(np.isnan(grad))
print("ok")
"""
    env = dict(os.environ, FGT_FAULT="launch")
    assert "ok" in _run_child(code, env)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device status")
def test_no_device_status(fgt):
    assert _call(fgt) == fgt.FGT_ERR_NODEVICE


def test_product_has_no_cpu_fallback():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "fgt_b200")
    for f in os.listdir(pkg):
        if f.endswith(".py"):
            txt = open(os.path.join(pkg, f)).read()
            assert "oracle" not in re.sub(r"#.*", "", txt).replace('"""', ""), f
