"""Benchmark of the B200 point FGT (pfgt) on the headline workload.

Workload: 3D, N = M = 1e7 points (sources = targets), 99% on the sphere of
radius 0.4 plus 1% uniform background, charges N(0,1), delta = 1e-4,
eps = 1e-6, potential + gradient at sources and targets (the delta=1e-4 cell
of the precision sweep).  A step is one pfgt call over the whole point set.
Metric: (N + M) evaluation points per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
  python bench.py --impl reference   (CPU arm: the oracle port on host cores)

Multi-GPU (torchrun): every rank runs an independent replica of the workload
(weak scaling, no data-path collective); the timed region is bracketed by
barriers and the max over ranks is reported.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "(N+M) pts/s, 3D N=1e7 eps=1e-6: mixed vs FP64 GPU path; rel err vs FP64 oracle"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="fgt", choices=["fgt", "reference"])
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--scale", type=float, default=1.0, help="fraction of N (tests only)")
    p.add_argument("--delta", type=float, default=1e-4)
    p.add_argument("--eps", type=float, default=1e-6)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-accuracy", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--profile-once", action="store_true",
                   help="one untimed step only (for ncu launch lists)")
    p.add_argument("--profile-config", type=int, default=5, choices=[1, 2, 3, 5],
                   help="configuration of the --profile-once step (--scale, and --delta/--eps "
                        "for configuration 3 and 5, apply)")
    p.add_argument("--sweep", default="cells", choices=["none", "cells", "all"],
                   help="also time the benchmark's other configurations: 'cells' = the "
                        "delta/eps cells of the sphere workload at eps=1e-6 plus configs 1-3, "
                        "'all' = every delta x eps cell")
    p.add_argument("--sweep-only", action="store_true", help="skip the headline extras")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                smax.append(float(f[2].split()[0]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


_PEAK_CACHE = {}


def flop_peak(dtype):
    """Measured SIMT peak: cuBLAS GEMM of the kernel's arithmetic type
    (TF32 off), best of 5 (TFLOP/s)."""
    import torch
    if dtype in _PEAK_CACHE:
        return _PEAK_CACHE[dtype]
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192 if dtype == torch.float32 else 4096
    x = torch.randn(n, n, dtype=dtype, device="cuda")
    y = torch.randn(n, n, dtype=dtype, device="cuda")
    for _ in range(2):
        x @ y
    best = 1e30
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        x @ y
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    v = 2.0 * n ** 3 / (best * 1e-3) / 1e12
    _PEAK_CACHE[dtype] = v
    return v


def ncu_traffic():
    """Per-launch DRAM traffic of the dominant kernels from the committed ncu
    summary (profiles/ncu_traffic.json), if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def roofline(a, stats, ms_phase):
    """Roofline of the dominant phase (measured with CUDA events on the
    launching stream inside the timed region)."""
    import torch
    names = {4: "form", 5: "translate", 6: "eval", 7: "direct"}
    flops = {4: stats["flops_form"], 6: stats["flops_eval"], 7: stats["flops_direct"]}
    dom = max(names, key=lambda i: ms_phase[i])
    ms = float(ms_phase[dom])
    tr = ncu_traffic().get(names[dom] + ("_" + a.precision), None)
    if dom == 5:
        bw, src = peaks()
        ach = stats["bytes_translate"] / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "kernel": names[dom], "achieved": ach, "peak": bw,
                "unit": "GB/s", "frac": ach / bw, "traffic": tr, "peak_source": src,
                "ms": ms}
    dt = torch.float32 if a.precision == "mixed" else torch.float64
    pk = flop_peak(dt)
    ach = flops[dom] / (ms * 1e-3) / 1e12
    return {"bound": "fp32" if a.precision == "mixed" else "fp64", "kernel": names[dom],
            "achieved": ach, "peak": pk, "unit": "TFLOP/s", "frac": ach / pk, "traffic": tr,
            "peak_source": "measured cuBLAS %s GEMM in bench.py (no tensor-core path: "
                           "no step is a dense contraction)" % ("FP32" if dt == torch.float32 else "FP64"),
            "ms": ms, "flops": flops[dom]}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def sample_window(src, frac, rng):
    """Points of the workload inside a cube around a sphere point holding
    about `frac` of them: same local density and tree structure, bounded
    size (the CPU baseline's sample)."""
    n = src.shape[0]
    c = src[rng.integers(n)]
    d = np.max(np.abs(src - c), axis=1)
    k = max(1000, int(frac * n))
    h = np.partition(d, k)[k]
    return np.nonzero(d <= h)[0]


def cpu_reference(cfg, target_s=10.0, frac=None):
    """Time the CPU restatement of the reference (FP64 C, OpenMP over boxes,
    its own ES-kernel NUFFT) on a spatial window of the workload, grown until
    one run takes about target_s; returns (pts/s, sample description, cores,
    frac used)."""
    from oracle import oracle as O
    rng = np.random.default_rng(1)
    src = cfg["sources"]
    frac = frac or 1e-3
    while True:
        idx = sample_window(src, frac, rng)
        s = src[idx]
        q = cfg["charge"][idx]
        t0 = time.perf_counter()
        out = O.pfgt(cfg["nd"], 3, cfg["delta"], cfg["eps"], 0, s, charge=q, ifpgh=cfg["ifpgh"],
                     targets=s.copy(), ifpghtarg=cfg["ifpghtarg"], nufft="spread")
        t = time.perf_counter() - t0
        if t >= 0.3 * target_s or frac >= 0.05:
            break
        frac = min(0.05, frac * max(2.0, min(8.0, target_s / max(t, 1e-3))))
    npts = 2 * len(idx)
    desc = (f"{len(idx)} sources + {len(idx)} targets (same points) inside a cube of the "
            f"workload, {t:.2f} s per run, nufft=spread")
    cpu_reference.last = (idx, out)
    cpu_reference.last_seconds = t
    return npts / t, desc, O.threads(), frac


def window_parity(F, cfg, prec, idx, ref_out, nexact=200):
    """The GPU path on the CPU baseline's window (same points, charges and
    parameters) against the restatement's output there, and both against the
    exact FP64 sum over the window's sources at `nexact` window points."""
    from oracle import oracle as O
    s = cfg["sources"][idx]
    q = cfg["charge"][idx]
    r = F.pfgt(cfg["nd"], 3, cfg["delta"], cfg["eps"], 0, s, charge=q, ifpgh=cfg["ifpgh"],
               targets=s.copy(), ifpghtarg=cfg["ifpghtarg"], precision=prec)
    out = {"points": int(len(idx)), "gpu_vs_restatement": {
        "pot": O.relerr(ref_out["pot"], r["pot"]), "grad": O.relerr(ref_out["grad"], r["grad"]),
        "pottarg": O.relerr(ref_out["pottarg"], r["pottarg"]),
        "gradtarg": O.relerr(ref_out["gradtarg"], r["gradtarg"])}}
    k = np.random.default_rng(3).choice(len(idx), min(nexact, len(idx)), replace=False)
    ex = O.direct_exact(cfg["nd"], 3, cfg["delta"], s, s[k], charge=q, ifpgh=2)
    out["vs_exact"] = {
        "sample": f"{len(k)} window points, FP64 direct sum over the window's sources (CPU)",
        "restatement": {"pot": O.relerr(ex["pot"], ref_out["pot"][k]),
                        "grad": O.relerr(ex["grad"], ref_out["grad"][k])},
        "gpu": {"pot": O.relerr(ex["pot"], r["pot"][k]),
                "grad": O.relerr(ex["grad"], r["grad"][k])}}
    return out


def _ptr(t):
    return None if t is None else t.data_ptr()


def exact_sample(F, dev, stream, cfg, pts_d, pgh):
    """FP64 direct sum over all sources (no cut-off; periodic: images
    |n_d| <= 1, enough for delta <= 1e-3 on the unit cell) at pts_d, by the
    library's all-pairs kernel."""
    import ctypes as C
    import itertools
    import torch
    n, nd, dim = pts_d.shape[0], cfg["nd"], cfg["dim"]
    ep = torch.zeros((n, nd), dtype=torch.float64, device=dev)
    eg = torch.zeros((n, dim, nd), dtype=torch.float64, device=dev)
    L = F.lib()
    f = L.fgt_direct_nomalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int,
                  C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                  C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p]
    src_d = cfg["_src_d"]
    q_d = cfg["_q_d"]
    shifts = [None]
    if cfg["iperiod"] == 1:
        shifts = [np.array(v, dtype=np.float64) * cfg["bs0"]
                  for v in itertools.product((-1.0, 0.0, 1.0), repeat=dim)]
    for sh in shifts:
        rc = f(nd, dim, cfg["delta"], 1e300,
               None if sh is None else sh.ctypes.data_as(C.c_void_p), src_d.shape[0],
               src_d.data_ptr(), 1, q_d.data_ptr(), 0, None, None, n, pts_d.data_ptr(), pgh,
               ep.data_ptr(), eg.data_ptr() if pgh >= 2 else None, None,
               C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError("fgt_direct_nomalloc failed: %d" % rc)
    torch.cuda.synchronize()
    return ep, eg


def run_cell(F, dev, stream, cfg, prec, steps, warmup, exact=None):
    """Time one configuration at one precision (device-resident inputs and
    outputs, CUDA events on the launching stream) and measure its relative
    l2 error at a sample of 1000 + 1000 points against the FP64 direct sum."""
    import ctypes as C
    import torch
    nd, dim = cfg["nd"], cfg["dim"]
    N = cfg["sources"].shape[0]
    has_t = cfg.get("targets") is not None
    M = cfg["targets"].shape[0] if has_t else 0
    if "_src_d" not in cfg:
        cfg["_src_d"] = torch.from_numpy(cfg["sources"]).to(dev)
        cfg["_q_d"] = torch.from_numpy(np.ascontiguousarray(cfg["charge"])).to(dev)
        cfg["_trg_d"] = torch.from_numpy(cfg["targets"]).to(dev) if has_t else None
    src_d, q_d, trg_d = cfg["_src_d"], cfg["_q_d"], cfg["_trg_d"]
    pgh, pght = cfg["ifpgh"], cfg["ifpghtarg"] if has_t else 0
    pot = torch.empty((N, nd), dtype=torch.float64, device=dev)
    grad = torch.empty((N, dim, nd), dtype=torch.float64, device=dev) if pgh >= 2 else None
    pt = torch.empty((max(M, 1), nd), dtype=torch.float64, device=dev)
    gt = torch.empty((max(M, 1), dim, nd), dtype=torch.float64, device=dev) if pght >= 2 else None
    st = F.FgtStats()
    o = F.FgtOpts()
    F.lib().fgt_opts_default(C.byref(o))
    o.precision = prec
    o.device_ptrs = 1
    o.device = dev.index
    o.stream = C.c_void_p(stream.cuda_stream)
    b0 = cfg.get("bs0", 1.0)
    c0 = cfg.get("cen0", [0.0] * 3)

    def step(opts):
        F.pfgt_device(opts, nd, dim, cfg["delta"], cfg["eps"], cfg["iperiod"], b0, c0, N,
                      src_d.data_ptr(), 1, q_d.data_ptr(), 0, None, None, pgh, pot.data_ptr(),
                      _ptr(grad), None, M, _ptr(trg_d), pght, pt.data_ptr() if M else None,
                      _ptr(gt), None)

    for _ in range(warmup):
        step(o)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step(o)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ot = F.FgtOpts()
    F.lib().fgt_opts_default(C.byref(ot))
    ot.precision, ot.device_ptrs, ot.device = prec, 1, dev.index
    ot.stream = C.c_void_p(stream.cuda_stream)
    ot.timing = 1
    ot.stats = C.pointer(st)
    step(ot)
    torch.cuda.synchronize()
    sd = st.as_dict()
    npts = N * (pgh > 0) + M * (pght > 0)
    out = {"precision": "fp64" if prec == F.PREC_FP64 else "mixed", "ms": ms,
           "value": npts / (ms * 1e-3), "unit": "pts/s", "steps": steps,
           "phases_ms": {k: round(float(v), 3) for k, v in zip(
               ["h2d", "tree", "sort_gather", "lists", "form", "translate", "eval", "direct",
                "scatter", "d2h", "total"], sd["ms"][:11])},
           "stats": {k: sd[k] for k in ("npwlevel", "nlevels", "npw", "n_form_boxes",
                                         "n_eval_boxes", "near_pairs", "spread_width")}}
    if exact is not None:
        i_s, x_sp, x_sg, i_t, x_tp, x_tg = exact
        rp = [(x_sp, pot[i_s])]
        rg = [(x_sg, grad[i_s])] if pgh >= 2 else []
        if M and pght >= 1:
            rp.append((x_tp, pt[i_t]))
            if pght >= 2:
                rg.append((x_tg, gt[i_t]))

        def rel(pairs):
            ref = torch.cat([r.reshape(-1) for r, _ in pairs])
            got = torch.cat([g.reshape(-1) for _, g in pairs])
            return float(torch.linalg.norm(ref - got) / torch.linalg.norm(ref))

        out["rel_l2"] = {"pot": rel(rp)}
        if rg:
            out["rel_l2"]["grad"] = rel(rg)
    out["_outputs"] = (pot, grad, pt if M else None, gt)
    return out


def exact_for(F, dev, stream, cfg, nsample=1000):
    import torch
    g = torch.Generator().manual_seed(7)
    N = cfg["sources"].shape[0]
    has_t = cfg.get("targets") is not None
    M = cfg["targets"].shape[0] if has_t else 0
    pgh = max(cfg["ifpgh"], cfg["ifpghtarg"] if has_t else 0)
    i_s = torch.randperm(N, generator=g)[:min(nsample, N)].to(dev)
    xs_p, xs_g = exact_sample(F, dev, stream, cfg, cfg["_src_d"][i_s].contiguous(), pgh)
    i_t, xt_p, xt_g = None, None, None
    if M:
        i_t = torch.randperm(M, generator=g)[:min(nsample, M)].to(dev)
        xt_p, xt_g = exact_sample(F, dev, stream, cfg, cfg["_trg_d"][i_t].contiguous(), pgh)
    return i_s, xs_p, xs_g, i_t, xt_p, xt_g


def sweep(a, F, dev, stream, W):
    """The benchmark's configurations besides the headline, each with the
    mixed path (where eps >= 1e-6, and for configuration 2 by its own
    definition) and the FP64 path side by side."""
    import torch
    cells = []
    plan = [("config1", W.config(1), None), ("config2", W.config(2), None),
            ("config3", W.config(3), None)]
    c5 = W.config(5)
    deltas = (1e-6, 1e-4, 1e-2, 1e-1)
    epss = (1e-3, 1e-6, 1e-9, 1e-12) if a.sweep == "all" else (1e-6,)
    for d in deltas:
        for e in epss:
            cfg = dict(c5)
            cfg["delta"], cfg["eps"] = d, e
            plan.append(("config5 delta=%g eps=%g" % (d, e), cfg, d))
    exact_cache = {}
    for name, cfg, dkey in plan:
        cfg = {k: v for k, v in cfg.items()}
        if dkey is not None:  # one device copy of the sphere workload for all cells
            for k in ("_src_d", "_q_d", "_trg_d"):
                if k in c5:
                    cfg[k] = c5[k]
        precs = [F.PREC_MIXED, F.PREC_FP64]
        if cfg["eps"] < 1e-6 and name != "config2":
            precs = [F.PREC_FP64]
        cell = {"name": name, "N": cfg["sources"].shape[0],
                "M": 0 if cfg.get("targets") is None else cfg["targets"].shape[0],
                "delta": cfg["delta"], "eps": cfg["eps"], "dim": cfg["dim"], "nd": cfg["nd"],
                "iperiod": cfg["iperiod"], "ifpgh": cfg["ifpgh"], "ifpghtarg": cfg["ifpghtarg"],
                "runs": []}
        try:
            for prec in precs:
                steps = max(2, min(a.steps, 5))
                r = run_cell(F, dev, stream, cfg, prec, steps, 2)
                if dkey is not None:
                    for k in ("_src_d", "_q_d", "_trg_d"):
                        c5[k] = cfg[k]
                key = (dkey, cfg["delta"]) if dkey is not None else name
                if key not in exact_cache:
                    exact_cache[key] = exact_for(F, dev, stream, cfg)
                ex = exact_cache[key]
                r2 = run_cell(F, dev, stream, cfg, prec, 1, 0, exact=ex)
                r["rel_l2"] = r2["rel_l2"]
                r.pop("_outputs", None)
                del r2
                cell["runs"].append(r)
            if len(cell["runs"]) == 2:
                cell["mixed_speedup"] = cell["runs"][1]["ms"] / cell["runs"][0]["ms"]
        except Exception as ex:  # keep the other cells
            cell["error"] = repr(ex)[:300]
        torch.cuda.synchronize()
        cells.append(cell)
        print("sweep:", json.dumps(cell), file=sys.stderr, flush=True)
    return cells


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from fgt_b200 import workloads as W
    cfg = W.config(5, scale=a.scale, delta=a.delta, eps=a.eps)
    npts = cfg["sources"].shape[0] + cfg["targets"].shape[0]
    config = {"workload": cfg["name"], "N": cfg["sources"].shape[0], "M": cfg["targets"].shape[0],
              "delta": cfg["delta"], "eps": cfg["eps"], "dim": 3, "nd": 1,
              "ifpgh": 2, "ifpghtarg": 2, "precision": a.precision,
              "l2": "inputs larger than L2 (240 MB coordinates per side)"}

    if a.impl == "reference":
        if rank != 0:
            return
        t0 = time.perf_counter()
        vals, secs = [], []
        sample = ""
        cores = 1
        frac = None
        # a step is one bounded sample of the workload (a spatial window of
        # it), so the whole run stays within a few minutes; ms_per_step is
        # the measured time of those sample steps, value their rate
        per_step = max(1.0, min(6.0, 90.0 / (a.warmup + a.steps)))
        for i in range(a.warmup + a.steps):
            v, sample, cores, frac = cpu_reference(cfg, target_s=per_step, frac=frac)
            if i >= a.warmup:
                vals.append(v)
                secs.append(cpu_reference.last_seconds)
        v = float(np.median(vals))
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "pts/s",
                "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": 1e3 * float(np.median(secs)),
                "step": "one bounded sample of the workload per step: " + sample,
                "full_workload_ms_at_this_rate": 1e3 * npts / v,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": v, "unit": "pts/s", "cores": cores, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": v, "unit": "pts/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "note": "reference Fortran build unavailable on this box (no Fortran "
                        "compiler, finufft, FFTW); the timed CPU code is the C restatement"}
        print(json.dumps(line))
        return

    import torch
    import fgt_b200 as F
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    prec = F.PREC_MIXED if a.precision == "mixed" else F.PREC_FP64
    if a.sweep_only:
        cells = sweep(a, F, dev, stream, W)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "sweep": cells}), flush=True)
        return

    # device-resident inputs and outputs (reference layouts, FP64)
    src_d = torch.from_numpy(cfg["sources"]).to(dev)
    trg_d = torch.from_numpy(cfg["targets"]).to(dev)
    q_d = torch.from_numpy(cfg["charge"]).to(dev)
    N, M = src_d.shape[0], trg_d.shape[0]
    pot_d = torch.empty((N, 1), dtype=torch.float64, device=dev)
    grad_d = torch.empty((N, 3, 1), dtype=torch.float64, device=dev)
    pt_d = torch.empty((M, 1), dtype=torch.float64, device=dev)
    gt_d = torch.empty((M, 3, 1), dtype=torch.float64, device=dev)
    st = F.FgtStats()
    import ctypes as C

    def opts(device_ptrs, timing):
        o = F.FgtOpts()
        F.lib().fgt_opts_default(C.byref(o))
        o.precision = prec
        o.device_ptrs = device_ptrs
        o.device = local
        o.stream = C.c_void_p(stream.cuda_stream)
        o.timing = 1 if timing else 0
        # statistics (device read-backs) only in the untimed phase pass
        o.stats = C.pointer(st) if timing else None
        return o

    od = opts(1, False)  # timed steps: no per-phase events
    odt = opts(1, True)  # phase breakdown, measured after the timed region

    def step_dev(o=None):
        F.pfgt_device(o or od, 1, 3, cfg["delta"], cfg["eps"], 0, 1.0, [0, 0, 0], N,
                      src_d.data_ptr(), 1, q_d.data_ptr(), 0, None, None, 2,
                      pot_d.data_ptr(), grad_d.data_ptr(), None, M, trg_d.data_ptr(), 2,
                      pt_d.data_ptr(), gt_d.data_ptr(), None)

    if a.profile_once:
        if a.profile_config == 5:
            step_dev()
        else:
            pc = W.config(a.profile_config, scale=a.scale)
            if a.profile_config == 3:
                pc["delta"], pc["eps"] = a.delta, a.eps
            run_cell(F, dev, stream, pc, prec, 1, 0)
        torch.cuda.synchronize()
        return

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def maxr(x):
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([x], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    for _ in range(a.warmup):
        step_dev()
    barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step_dev()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    ms = maxr(e0.elapsed_time(e1) / a.steps)
    value = world * npts / (ms * 1e-3)
    # per-phase CUDA-event times of the same call (untimed region)
    ms_phase = np.zeros(12)
    nph = 3
    for _ in range(nph):
        step_dev(odt)
        ms_phase += np.array(st.ms[:12])
    ms_phase /= nph
    stats = st.as_dict()

    # relative l2 error against an FP64 direct summation (all N sources, no
    # cut-off) at a sample of evaluation points, computed on the GPU by the
    # library's FP64 all-pairs kernel, independent of the fast path
    def exact_at(pts_d):
        n = pts_d.shape[0]
        ep = torch.zeros((n, 1), dtype=torch.float64, device=dev)
        eg = torch.zeros((n, 3, 1), dtype=torch.float64, device=dev)
        L = F.lib()
        f = L.fgt_direct_nomalloc
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_int,
                      C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                      C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_void_p]
        rc = f(1, 3, cfg["delta"], 1e300, None, N, src_d.data_ptr(), 1, q_d.data_ptr(), 0,
               None, None, n, pts_d.data_ptr(), 2, ep.data_ptr(), eg.data_ptr(), None,
               C.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError("fgt_direct_nomalloc failed: %d" % rc)
        torch.cuda.synchronize()
        return ep, eg

    def rel(ref, got):
        ref = ref.reshape(-1)
        return float(torch.linalg.norm(ref - got.reshape(-1)) / torch.linalg.norm(ref))

    acc = None
    if not a.no_accuracy:
        g = torch.Generator().manual_seed(7)
        ns_s = min(1000, N)
        ns_t = min(1000, M)
        i_s = torch.randperm(N, generator=g)[:ns_s].to(dev)
        i_t = torch.randperm(M, generator=g)[:ns_t].to(dev)
        xs_p, xs_g = exact_at(src_d[i_s].contiguous())
        xt_p, xt_g = exact_at(trg_d[i_t].contiguous())

        def errs():
            return {"pot": rel(torch.cat([xs_p, xt_p]), torch.cat([pot_d[i_s], pt_d[i_t]])),
                    "grad": rel(torch.cat([xs_g, xt_g]), torch.cat([grad_d[i_s], gt_d[i_t]]))}

        acc = {"reference": "FP64 direct sum over all sources (no cut-off), GPU all-pairs kernel",
               "sample": f"{ns_s} sources + {ns_t} targets", "rel_l2": errs()}
        if rank == 0 and world == 1 and not a.no_cpu:
            # the GPU all-pairs reference itself checked by the CPU oracle's
            # exact sum over all N sources at a few of the sampled points
            from oracle import oracle as O
            kx = 32
            pts = src_d[i_s[:kx]].cpu().numpy()
            t0 = time.perf_counter()
            ce = O.direct_exact(1, 3, cfg["delta"], cfg["sources"], pts, charge=cfg["charge"],
                                ifpgh=2)
            acc["cpu_exact_crosscheck"] = {
                "points": kx, "seconds": round(time.perf_counter() - t0, 2),
                "gpu_allpairs_vs_cpu_exact": {
                    "pot": O.relerr(ce["pot"], xs_p[:kx].cpu().numpy()),
                    "grad": O.relerr(ce["grad"], xs_g[:kx].cpu().numpy())},
                "fast_path_vs_cpu_exact": {
                    "pot": O.relerr(ce["pot"], pot_d[i_s[:kx]].cpu().numpy()),
                    "grad": O.relerr(ce["grad"], grad_d[i_s[:kx]].cpu().numpy())}}
        # the FP64 GPU path side by side: time and error on the same workload
        if world == 1 and a.precision == "mixed":
            mixed_out = [t.clone() for t in (pot_d, grad_d, pt_d, gt_d)]
            o64 = opts(1, False)
            o64.precision = F.PREC_FP64
            for _ in range(2):
                step_dev(o64)
            torch.cuda.synchronize()
            k64 = max(2, min(a.steps, 5))
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            g0.record(stream)
            for _ in range(k64):
                step_dev(o64)
            g1.record(stream)
            torch.cuda.synchronize()
            ms64 = g0.elapsed_time(g1) / k64
            both = list(zip(mixed_out, (pot_d, grad_d, pt_d, gt_d)))
            acc["fp64_path"] = {"value": npts / (ms64 * 1e-3), "unit": "pts/s",
                                "ms_per_step": ms64, "steps": k64, "rel_l2": errs(),
                                "mixed_speedup": ms64 / ms,
                                "mixed_vs_fp64_rel_l2_all_points": {
                                    "pot": rel(torch.cat([b.reshape(-1) for _, b in both[0::2]]),
                                               torch.cat([m.reshape(-1) for m, _ in both[0::2]])),
                                    "grad": rel(torch.cat([b.reshape(-1) for _, b in both[1::2]]),
                                                torch.cat([m.reshape(-1) for m, _ in both[1::2]]))}}
            del mixed_out, both
            step_dev()  # leave the mixed results in the output buffers
            torch.cuda.synchronize()

    # end to end through the public API with pinned host buffers
    e2e = None
    if not a.no_e2e:
        hs = torch.from_numpy(cfg["sources"]).pin_memory()
        ht = torch.from_numpy(cfg["targets"]).pin_memory()
        hq = torch.from_numpy(cfg["charge"]).pin_memory()
        hp = torch.empty((N, 1), dtype=torch.float64).pin_memory()
        hg = torch.empty((N, 3, 1), dtype=torch.float64).pin_memory()
        hpt = torch.empty((M, 1), dtype=torch.float64).pin_memory()
        hgt = torch.empty((M, 3, 1), dtype=torch.float64).pin_memory()
        oh = opts(0, False)

        def step_host():
            F.pfgt_device(oh, 1, 3, cfg["delta"], cfg["eps"], 0, 1.0, [0, 0, 0], N,
                          hs.data_ptr(), 1, hq.data_ptr(), 0, None, None, 2, hp.data_ptr(),
                          hg.data_ptr(), None, M, ht.data_ptr(), 2, hpt.data_ptr(),
                          hgt.data_ptr(), None)

        for _ in range(max(1, a.warmup // 2)):
            step_host()
        barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(a.steps):
            step_host()
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = maxr(f0.elapsed_time(f1) / a.steps)
        h2d = (N * 3 + M * 3 + N) * 8
        d2h = (N * 4 + M * 4) * 8
        e2e = {"value": world * npts / (ms_e2e * 1e-3), "unit": "pts/s",
               "ms_per_step": ms_e2e, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    # reusable plan on the same workload: the tree, lists and sorted offsets
    # are built once; each step is fgt_plan_execute with the charges
    plan = None
    if rank == 0 and world == 1:
        L = F.lib()
        L.fgt_plan_create.restype = C.c_void_p
        L.fgt_plan_execute.restype = C.c_int
        op = opts(1, False)
        st_c = C.c_int(0)
        b0p, c0p = C.c_double(1.0), np.zeros(3)
        h = L.fgt_plan_create(C.byref(op), 1, 3, C.c_double(cfg["delta"]), C.c_double(cfg["eps"]),
                              0, C.byref(b0p), c0p.ctypes.data_as(C.c_void_p), N,
                              C.c_void_p(src_d.data_ptr()), M, C.c_void_p(trg_d.data_ptr()),
                              C.byref(st_c))
        if not h:
            raise RuntimeError("fgt_plan_create failed: %d" % st_c.value)
        ref_pot = pot_d.clone()
        outp = [torch.empty_like(t) for t in (pot_d, grad_d, pt_d, gt_d)]

        def step_plan():
            rc = L.fgt_plan_execute(C.c_void_p(h), 1, C.c_void_p(q_d.data_ptr()), 0, None, None, 2,
                                    C.c_void_p(outp[0].data_ptr()), C.c_void_p(outp[1].data_ptr()),
                                    None, 2, C.c_void_p(outp[2].data_ptr()),
                                    C.c_void_p(outp[3].data_ptr()), None)
            if rc != 0:
                raise RuntimeError("fgt_plan_execute failed: %d" % rc)

        for _ in range(max(1, a.warmup)):
            step_plan()
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(a.steps):
            step_plan()
        p1.record(stream)
        torch.cuda.synchronize()
        msp = p0.elapsed_time(p1) / a.steps
        plan = {"ms_per_execute": msp, "value": npts / (msp * 1e-3), "unit": "pts/s",
                "pot_rel_diff_vs_call": float(torch.linalg.norm(outp[0] - ref_pot) /
                                              torch.linalg.norm(ref_pot)),
                "note": "fgt_plan_execute on the same points (tree, lists, offsets reused)"}
        L.fgt_plan_destroy(C.c_void_p(h))
        del outp, ref_pot

    # batched workload: 512 independent instances through fgt_pfgt_batch
    # (device-resident inputs), against a loop of single calls
    batch = None
    if rank == 0 and world == 1 and not a.no_batch:
        inst = W.batch_instances()
        L = F.lib()
        L.fgt_pfgt_batch.restype = C.c_int
        arr = (F.FgtInstance * len(inst))()
        keepb = []
        for x, kw in zip(arr, inst):
            s_ = torch.from_numpy(kw["sources"]).to(dev)
            q_ = torch.from_numpy(kw["charge"]).to(dev)
            p_ = torch.empty((s_.shape[0], 1), dtype=torch.float64, device=dev)
            b0, c0 = np.array([1.0]), np.zeros(3)
            keepb.append((s_, q_, p_, b0, c0))
            x.nd, x.dim, x.delta, x.eps, x.iperiod = 1, 3, kw["delta"], kw["eps"], 0
            x.bs0, x.cen0 = F._ptr(b0), F._ptr(c0)
            x.ns, x.sources, x.ifcharge, x.charge = s_.shape[0], s_.data_ptr(), 1, q_.data_ptr()
            x.ifpgh, x.pot = 1, p_.data_ptr()
        ob = F.FgtOpts()
        L.fgt_opts_default(C.byref(ob))
        ob.device_ptrs = 1
        nb_pts = sum(x["sources"].shape[0] for x in inst)
        L.fgt_pfgt_batch(C.byref(ob), len(inst), arr, 0)
        torch.cuda.synchronize()
        tb = []
        for _ in range(3):
            t0 = time.perf_counter()
            rc = L.fgt_pfgt_batch(C.byref(ob), len(inst), arr, 0)
            torch.cuda.synchronize()
            tb.append(time.perf_counter() - t0)
            if rc != 0:
                raise RuntimeError("fgt_pfgt_batch failed: %d" % rc)
        t0 = time.perf_counter()
        L.fgt_pfgt_batch(C.byref(ob), len(inst), arr, 1)
        torch.cuda.synchronize()
        t1 = time.perf_counter() - t0
        batch = {"workload": "512 independent 3D instances, N log-uniform in [1e3, 1e5] "
                             "(sources = targets), half uniform / half sphere, delta "
                             "log-uniform in [1e-5, 1e-2], eps in {1e-3, 1e-6}, pot only",
                 "points": nb_pts, "value": nb_pts / min(tb), "unit": "pts/s",
                 "ms": 1e3 * min(tb), "timing": "host wall clock around the synchronous call",
                 "sequential_value": nb_pts / t1,
                 "note": "default worker count; sequential = the same call with one worker"}
        del keepb

    cells = None
    if a.sweep != "none" and world == 1:
        del src_d, trg_d, q_d, pot_d, grad_d, pt_d, gt_d
        torch.cuda.empty_cache()
        cells = sweep(a, F, dev, stream, W)
    roof = roofline(a, stats, ms_phase)
    rho = ncu_traffic().get("translate_l2_read_miss_fraction")
    if rho is not None:
        roof["translate_rho"] = rho  # fraction of translation reads that miss L2 (ncu)
    if roof.get("traffic") is not None:
        roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                                  "of the kernel on the 0.3-scale workload, scaled to this size "
                                  "by points and boxes (profiles/ncu_traffic.json)")
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        v, desc, cores, _ = cpu_reference(cfg, target_s=12.0)
        cpu = {"value": v, "unit": "pts/s", "cores": cores, "kind": "port", "sample": desc}
        widx, wout = cpu_reference.last
        cpu["window_parity"] = window_parity(F, cfg, prec, widx, wout)
    line = {"metric": METRIC, "value": value, "unit": "pts/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if a.precision == "mixed" else "f64", "data": "synthetic",
            "config": config, "clocks": clocks, "e2e": e2e, "roofline": roof,
            "cpu_baseline": cpu, "accuracy": acc, "batch": batch, "plan": plan, "sweep": cells,
            "gpu_launches": int(stats["n_kernel_launches"]) * a.steps,
            "phases_ms": {k: round(float(v), 4) for k, v in zip(
                ["h2d", "tree", "sort_gather", "lists", "form", "translate", "eval", "direct",
                 "scatter", "d2h", "total"], ms_phase[:11])},
            "stats": {k: stats[k] for k in ("nlevels", "nboxes", "npwlevel", "npw",
                                             "n_form_boxes", "n_eval_boxes", "n_eval_nufft",
                                             "n_translations", "spread_width", "grid_cells",
                                             "near_pairs", "pts_form", "pts_eval_nufft",
                                             "pts_eval_modal", "flops_form", "flops_eval",
                                             "flops_direct", "bytes_translate")}}
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
