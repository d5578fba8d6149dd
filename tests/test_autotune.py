"""Autotuner (fgt_opts.autotune): a tuning run times the strength-dependent
part of a call with each candidate modal-evaluation threshold (and batches
with each worker count), keeps the fastest in the on-disk cache named by
FGT_TUNE_CACHE, and later calls of the same problem class take it from
there.  Results equal the untuned call's to the arithmetic's rounding."""
import ctypes as C

import numpy as np
import pytest

from conftest import relerr
from fgt_b200 import workloads as W


def test_autotune_is_off_by_default(fgt):
    o = fgt.FgtOpts()
    fgt.lib().fgt_opts_default(C.byref(o))
    assert o.autotune == 0 and o.root_level == -1 and o.small_eval == -1


@pytest.mark.gpu
def test_tuning_run_fills_the_cache_and_later_calls_use_it(fgt, tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("FGT_TUNE_CACHE", str(cache))
    cfg = W.config(5, scale=0.004, delta=1e-3, eps=1e-6)
    kw = {k: v for k, v in cfg.items() if k != "name"}
    plain = fgt.pfgt(precision=fgt.PREC_MIXED, stats=True, **kw)
    assert plain["stats"]["tuned"] == 0 and plain["stats"]["small_eval_used"] == 48
    tuned = fgt.pfgt(precision=fgt.PREC_MIXED, stats=True, autotune=2, **kw)
    assert tuned["stats"]["tuned"] == 1
    se = tuned["stats"]["small_eval_used"]
    assert se in (0, 16, 32, 48, 64, 96, 128)
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and lines[0].startswith("pfgt/v1 dim=3 fp32") and lines[0].endswith(" %d" % se)
    for f in ("pot", "grad", "pottarg", "gradtarg"):
        assert relerr(plain[f], tuned[f]) < 1e-6, f
    again = fgt.pfgt(precision=fgt.PREC_MIXED, stats=True, autotune=1, **kw)
    assert again["stats"]["tuned"] == 1 and again["stats"]["small_eval_used"] == se
    assert len(cache.read_text().splitlines()) == 1  # no second tuning run
    # another problem class (FP64 arithmetic) misses the cache: defaults
    other = fgt.pfgt(precision=fgt.PREC_FP64, stats=True, autotune=1, **kw)
    assert other["stats"]["tuned"] == 0 and other["stats"]["small_eval_used"] == 48


@pytest.mark.gpu
def test_batch_worker_count_is_tuned(fgt, tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("FGT_TUNE_CACHE", str(cache))
    insts = W.batch_instances(count=24, nmin=500, nmax=3000)
    ref = fgt.pfgt_batch(insts)
    got = fgt.pfgt_batch(insts, autotune=2)
    assert any(l.startswith("batch/v1 ") for l in cache.read_text().splitlines())
    for a, b in zip(ref, got):
        assert relerr(a["pot"], b["pot"]) < 1e-6
