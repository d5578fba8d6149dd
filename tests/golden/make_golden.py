"""Generates the golden fixtures of tests/golden/ from the oracle.

The reference (Fortran + finufft) cannot be built in this environment and
ships no golden vectors, so the fixtures record the restatement's outputs on
small seeded inputs (the reference test's point scenarios and the benchmark
distributions).  Their values are pinned independently by
tests/test_oracle.py against the exact FP64 Gauss transform.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fgt_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    rng = np.random.default_rng(20261203)
    cases = {
        "wiggly2d": dict(nd=1, dim=2, delta=1e-3, eps=1e-6, iperiod=0,
                         sources=W.wiggly_curve(rng, 3000, 2), ifpgh=2,
                         targets=rng.uniform(0, 1, (400, 2)), ifpghtarg=2, bs0=1.0, cen0=[0, 0]),
        "uniform3d_cfg1": dict(nd=1, dim=3, delta=1e-4, eps=1e-6, iperiod=0,
                               sources=W.uniform(rng, 4000, 3), ifpgh=1,
                               targets=np.zeros((0, 3)), ifpghtarg=0, bs0=1.0, cen0=[0, 0, 0]),
        "pw3d_eps1e-3": dict(nd=1, dim=3, delta=1e-2, eps=1e-3, iperiod=0,
                             sources=W.uniform(rng, 6000, 3), ifpgh=2,
                             targets=np.zeros((0, 3)), ifpghtarg=0, bs0=1.0, cen0=[0, 0, 0]),
        "periodic2d_nd2": dict(nd=2, dim=2, delta=1e-4, eps=1e-6, iperiod=1,
                               sources=W.uniform(rng, 5000, 2), ifpgh=2,
                               targets=np.zeros((0, 2)), ifpghtarg=0, bs0=1.0, cen0=[0, 0]),
    }
    for name, c in cases.items():
        n = c["sources"].shape[0]
        c["charge"] = rng.uniform(-1, 1, (n, c["nd"]))
        kw = dict(charge=c["charge"], ifpgh=c["ifpgh"], bs0=c["bs0"], cen0=c["cen0"])
        if c["targets"].shape[0]:
            kw["targets"] = c["targets"]
            kw["ifpghtarg"] = c["ifpghtarg"]
        r = O.pfgt(c["nd"], c["dim"], c["delta"], c["eps"], c["iperiod"], c["sources"], **kw)
        out = {k: np.asarray(v) for k, v in c.items()}
        for f in ("pot", "grad", "pottarg", "gradtarg"):
            if f in r:
                out[f] = r[f]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
