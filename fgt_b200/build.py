"""Builds the CUDA library fgt_b200/libfgt_b200.so for sm_100a (in-tree).

Each csrc/*.cu is compiled to an object with nvcc (in parallel, rebuilt when
the source or any header is newer), then linked into one shared library that
exports the C ABI of include/fgt_b200.h.  build(check=True) makes the
FGT_CHECK variant libfgt_b200_check.so (device bounds checks that record a
failing site and skip the access; the call then returns FGT_ERR_CHECK).
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfgt_b200.so")
OBJ_CHECK = os.path.join(HERE, "_build_check")
LIB_CHECK = os.path.join(HERE, "libfgt_b200_check.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", os.path.join(ROOT, "include")]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src, extra, objdir=OBJ):
    obj = os.path.join(objdir, os.path.basename(src).replace(".cu", ".o"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj, None
    cmd = [nvcc()] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "FAILED: " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(verbose=False, extra=None, check=False):
    """Compile and link; returns the library path (check: the FGT_CHECK
    variant, objects and library kept apart from the normal build)."""
    extra = list(extra or []) + (["-DFGT_CHECK=1"] if check else [])
    objdir, lib = (OBJ_CHECK, LIB_CHECK) if check else (OBJ, LIB)
    os.makedirs(objdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        res = list(ex.map(lambda s: _compile(s, extra, objdir), srcs))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("\n".join(errs))
    objs = [o for o, _ in res]
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: " + r.stdout + r.stderr)
    if verbose:
        print("built", lib)
    return lib


if __name__ == "__main__":
    args = sys.argv[1:]
    chk = "--check" in args
    build(verbose=True, extra=[a for a in args if a != "--check"], check=chk)
