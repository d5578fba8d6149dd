"""FGT_LOG=1: one JSON line per pfgt call on stderr (tree and list sizes,
per-phase device times, achieved rates); silent without it."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CALL = r"""
import numpy as np
import fgt_b200 as F
from fgt_b200 import workloads as W
rng = np.random.default_rng(3)
src = W.gaussian_clusters(rng, 20000, 3, ncl=4)
q = rng.standard_normal((20000, 1))
trg = W.uniform(rng, 2000, 3)
for prec in (F.PREC_MIXED, F.PREC_FP64):
    F.pfgt(nd=1, dim=3, delta=3e-3, eps=1e-6, iperiod=0, sources=src, charge=q, ifpgh=2,
           targets=trg, ifpghtarg=2, precision=prec)
"""


def _run(log):
    env = dict(os.environ)
    env.pop("FGT_LOG", None)
    if log:
        env["FGT_LOG"] = "1"
    r = subprocess.run([sys.executable, "-c", CALL], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stderr.splitlines() if l.startswith('{"fgt"')]


@pytest.mark.gpu
def test_fgt_log_lines():
    lines = _run(True)
    assert [l["precision"] for l in lines] == ["mixed", "fp64"]
    for l in lines:
        assert (l["ns"], l["nt"], l["nd"], l["dim"]) == (20000, 2000, 1, 3)
        assert l["nboxes"] > 0 and l["n_form_boxes"] > 0 and l["near_pairs"] > 0
        assert l["kernel_launches"] > 0
        ms = l["ms"]
        assert set(ms) == {"h2d", "tree", "sort_gather", "lists", "form", "translate", "eval",
                           "direct", "scatter", "d2h", "total"}
        assert ms["total"] > 0 and ms["tree"] > 0 and ms["eval"] > 0
        assert l["tflops"]["direct"] > 0
    assert _run(False) == []
