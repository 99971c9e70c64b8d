"""Benchmark of the all-pairs ML Jacquard estimator on B200.

Workload (one step): every pair of a synthetic cohort of N=1024 samples x
M=100,000 biallelic sites (REF frequency ~ Beta(0.5,0.5) clipped to
[0.05,0.95], Hardy-Weinberg genotypes, 2% of calls missing, 64 each of
parent-offspring, full-sib, half-sib and first-cousin pairs planted): allele
frequencies, site filtering and packing, then the SQP of all 524,800 pairs
(523,776 off-diagonal + 1,024 self).  The metric counts off-diagonal pairs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kestrel_b200|reference]
                  [--precision fp32c|fp64] [--samples N] [--sites M]

`value` is device-timed (CUDA events inside the library on its stream) with the
genotypes already in HBM; `e2e` runs the public C ABI from host buffers
(upload, estimation, copy of all rows back) each step.  Under torchrun each rank
runs the full workload on its own GPU (pairs are independent; no collective on
the data path), so scaling is weak and `value` sums the ranks.
"""
from __future__ import annotations

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

METRIC = "all-pairs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kestrel_b200", choices=["kestrel_b200", "reference"])
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--samples", type=int, default=1024)
    ap.add_argument("--sites", type=int, default=100_000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 form's measurement")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--slots", type=int, default=0, help="pairs in flight per wave (0 = automatic)")
    ap.add_argument("--multi-sites", type=int, default=0,
                    help="gt-cls, ml-multi: tri- and tetra-allelic sites beside the biallelic ones")
    ap.add_argument("--pass-bps", type=int, default=0, help="site-pass blocks per SM (0 = automatic)")
    ap.add_argument("--workload", default="allpairs",
                    choices=["allpairs", "batch", "inbred", "serving", "gt-cls", "gl-soft", "ml-multi"],
                    help="allpairs: N x M all pairs (the headline); batch: 8 uneven cohorts in one "
                         "launch; inbred: N=512 x M=50k inbred stress; serving: panel + Poisson "
                         "query stream (p50/p99 latency)")
    ap.add_argument("--requests", type=int, default=64, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=200.0, help="serving: Poisson arrival rate (requests/s)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, pg, device: str) -> float:
    """The largest of every rank's value (one all-reduce; every rank calls it in
    the same order).  pg is torch.distributed or None for one process; device is
    where the reduction tensor lives (a CUDA device for NCCL, "cpu" for gloo)."""
    if pg is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(pairs_per_rank: int, world: int, ms_per_step: float) -> float:
    """Pairs per second of the whole job: every rank runs its own replica of the
    workload, timed by the slowest rank."""
    return world * pairs_per_rank / (ms_per_step * 1e-3)


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"])
    except Exception:
        return 6650.0


def workload_config(n, m):
    """The config dict of the all-pairs workload, the same in both arms."""
    return {"workload": f"all pairs of N={n} x M={m} (planted PO/FS/HS/FC)",
            "samples": n, "sites": m, "pairs": n * (n - 1) // 2, "self_pairs": n,
            "l2": "GPU arm: 256 MB buffer written between steps; the CPU arm has no GPU work"}


def cpu_baseline(codes, planted, seconds, threads=0, keep_rows=False):
    """The oracle (the reference's ML path restated in C, FP64, all host
    threads) on a bounded sample of this workload's pairs; pairs/s.  With
    keep_rows, also returns the sampled pairs and the oracle's rows for them."""
    from oracle import pyoracle
    p, q, keep = pyoracle.site_frequencies(codes)
    rng = np.random.default_rng(123)
    n = codes.shape[0]
    cores = threads or os.cpu_count()

    def sample(k):
        xs = rng.integers(0, n, k)
        ys = rng.integers(0, n, k)
        return np.stack([np.minimum(xs, ys), np.maximum(xs, ys)], 1)

    k = max(2 * cores, 16)
    t0 = time.perf_counter()
    pyoracle.relatedness_pairs(codes, p, q, keep, sample(k), threads=threads)
    dt = time.perf_counter() - t0
    k2 = int(max(k, min(200_000, k * max(1.0, (seconds - dt) / max(dt, 1e-3)))))
    pairs = sample(k2)
    t0 = time.perf_counter()
    rows = pyoracle.relatedness_pairs(codes, p, q, keep, pairs, threads=threads)
    dt2 = time.perf_counter() - t0
    out = {"value": k2 / dt2, "unit": "pairs/s", "cores": cores, "kind": "port",
           "sample": f"{k2} random pairs of the {n} x {codes.shape[1]} cohort "
                     f"(oracle FP64 restatement, OpenMP over {cores} threads, {dt2:.1f} s)"}
    if keep_rows:
        return out, pairs, rows, (p, q, keep)
    return out


def error_vs_oracle(gpu_rows, codes, planted, pairs, ref_rows, freqs):
    """Largest errors of the GPU rows against the FP64 oracle over the
    sampled pairs of the CPU leg plus every planted pair (run after the timed
    region): Delta and kinship over pairs whose oracle log10 condition
    estimate is below 15, the objective (relative) over all of them, and the
    pairs whose condition flag (log10 cond > 15) differs."""
    import kestrel_b200 as kb
    from oracle import pyoracle
    p, q, keep = freqs
    pl = np.array([(a, b) for a, b, _, _ in planted], dtype=np.int64).reshape(-1, 2)
    if len(pl):
        pairs = np.concatenate([pairs, pl])
        ref_rows = np.concatenate([ref_rows, pyoracle.relatedness_pairs(codes, p, q, keep, pl)])
    n = codes.shape[0]
    x, y = pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64)
    idx = x * n - x * (x - 1) // 2 + (y - x)          # row of (x, y) in the reference's order
    g = gpu_rows[idx]
    assert np.array_equal(g["x"].astype(np.int64), x) and np.array_equal(g["y"].astype(np.int64), y)
    lc_ref = np.log10(ref_rows["cond"])
    below = np.isfinite(lc_ref) & (lc_ref < 15)
    dd = np.abs(g["jacquard"] - ref_rows["jacquard"]).max(1)
    dk = np.abs(g["jacquard"] @ kb.KINSHIP_VECTOR - ref_rows["jacquard"] @ kb.KINSHIP_VECTOR)
    do = np.abs(g["obj"] - ref_rows["obj"]) / np.abs(ref_rows["obj"])
    flag = (np.log10(g["cond"]) > 15) != (lc_ref > 15)
    exact = below & (lc_ref < 13)
    return {"pairs": int(len(pairs)), "planted": int(len(pl)), "compared": int(below.sum()),
            "max_abs_delta_err": float(dd[below].max(initial=0)),
            "max_abs_kinship_err": float(dk[below].max(initial=0)),
            "max_rel_objective_err": float(do.max(initial=0)),
            "cond_flag_disagreements": int(np.sum(flag & exact)),
            "cond_13_15": {"pairs": int(np.sum(below & ~exact)), "flag_disagreements": int(np.sum(flag & below & ~exact))},
            "bar": "Delta and kinship <= 1e-5 absolute, objective <= 1e-6 relative on pairs with oracle "
                   "log10 cond < 15; condition flag equal where it is < 13",
            "oracle": "FP64 C restatement of the reference's ML path"}


def run_reference(args, codes, planted):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    n = codes.shape[0]
    pairs_per_step = n * (n - 1) // 2
    for _ in range(args.warmup):
        cpu_baseline(codes, planted, min(3.0, args.cpu_seconds / 5))
    vals = []
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(codes, planted, args.cpu_seconds / max(1, args.steps))
        vals.append(cb["value"])
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": pairs_per_step / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": workload_config(n, int(codes.shape[1])),
            "cpu_baseline": dict(cb, value=v),
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batch(args, local):
    """Eight cohorts of uneven N, M and missingness in one launch: timed with
    the default launch shape and with the one kg_autotune picks on a sample of
    the largest cohort, the two alternating step by step (both reported; the
    line's value is the default shape's, the tuned shape's beside it)."""
    import kestrel_b200 as kb
    from kestrel_b200 import synth
    cohorts = synth.config2()
    pairs = sum(c.codes.shape[0] * (c.codes.shape[0] - 1) // 2 for c in cohorts)
    import torch
    est = kb.Estimator(device=local, precision=args.precision)
    est.set_launch(args.slots, args.pass_bps)
    # page-locked genotypes and row buffers, reused by every call (uploads
    # from pageable memory vary by a few hundred ms from call to call)
    inputs = [(torch.from_numpy(c.codes).pin_memory().numpy(),) for c in cohorts]
    outs = [torch.empty(c.codes.shape[0] * (c.codes.shape[0] + 1) // 2 * kb.OUTPUT_DTYPE.itemsize,
                        dtype=torch.uint8, pin_memory=True).numpy().view(kb.OUTPUT_DTYPE) for c in cohorts]

    def run_once():
        t0 = time.perf_counter()
        est.relatedness_batch(inputs, out=outs)
        return time.perf_counter() - t0, est.run_stats()

    # the default shape first, for the warm-up and the tuner's sample
    for _ in range(max(1, args.warmup)):
        est.relatedness_batch(inputs, out=outs)
    default_shape = est.launch()
    big = max(cohorts, key=lambda c: c.codes.shape[0])
    est.load(big.codes)
    t0 = time.perf_counter()
    est.autotune()
    t_tune = time.perf_counter() - t0
    shape = est.launch()

    def apply(sh):
        est.set_launch(args.slots, sh["blocks_per_sm"] or args.pass_bps)
        est.set_work_unit(sh["unit_entries"])

    # the two shapes alternate step by step, so that clock and power drift
    # over the run falls on both alike (the tuner leaves the divisor of the
    # pairs in flight alone for a cohort this large, so the two differ at
    # most in blocks per SM and the work unit); a change of shape rebuilds
    # the engine's buffers and graphs, so each shape's timed call follows an
    # untimed one
    runs = {"default": ([], []), "tuned": ([], [])}
    st = None
    for _ in range(max(1, args.steps)):
        for name, sh in (("default", default_shape), ("tuned", shape)):
            apply(sh)
            est.relatedness_batch(inputs, out=outs)
            dt, st = run_once()
            runs[name][0].append(dt)
            runs[name][1].append(st["pair_kernel_ms"])
    # the median step: one host stall (page faults, another process) does
    # not move it
    t_default, w_default = float(np.median(runs["default"][0])), float(np.median(runs["default"][1]))
    tw, w_tuned = float(np.median(runs["tuned"][0])), float(np.median(runs["tuned"][1]))
    est.close()
    waves_ms = [w_default]
    return {"metric": "all-pairs/s, 8 uneven cohorts in one launch", "value": pairs / t_default,
            "unit": "pairs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_default * 1e3,
            "higher_is_better": True, "dtype": "f32" if args.precision == "fp32c" else "f64",
            "data": "synthetic",
            "config": {"workload": "cohorts N=" + "/".join(str(c.codes.shape[0]) for c in cohorts) +
                                   " x M=" + "/".join(str(c.codes.shape[1]) for c in cohorts) +
                                   ", per-sample missingness U(0, 0.2)", "pairs": pairs},
            "timing": "host wall clock around kg_relatedness_batch (uploads from page-locked memory, "
                      "preparation, waves, rows back into page-locked buffers), median of the steps; default and "
                      "tuned shapes alternate",
            "waves_ms": float(np.mean(waves_ms)), "waves_pairs_per_s": pairs / (np.mean(waves_ms) * 1e-3),
            "autotune": {"shape": shape, "tune_s": t_tune, "default_pairs_per_s": pairs / t_default,
                         "default_waves_ms": w_default, "tuned_pairs_per_s": pairs / tw, "tuned_waves_ms": w_tuned,
                         "note": "0 = the default (occupancy limit, 32768-entry units, a fifth of the pairs in "
                                 "flight); tuned on about 131,072 pairs of the 2048 x 100000 cohort"},
            "stats": {k: st[k] for k in ("gh_passes", "fp64_pairs", "waves", "slots", "nonconverged")}}


def run_inbred(args, local):
    """N=512 x M=50k with 128 inbred samples, 32 identical-inbred pairs and a
    low-information block (ill-conditioned Hessians)."""
    import kestrel_b200 as kb
    from kestrel_b200 import synth
    co = synth.config3()
    n = co.codes.shape[0]
    pairs = n * (n - 1) // 2
    est = kb.Estimator(device=local, precision=args.precision)
    est.set_launch(args.slots, args.pass_bps)
    est.load(co.codes)
    for _ in range(max(1, args.warmup)):
        est.relatedness()
    dev = []
    for _ in range(max(1, args.steps)):
        rows = est.relatedness()
        st = est.run_stats()
        dev.append(st["device_ms"])
    est.close()
    t = float(np.mean(dev))
    cond = rows["cond"]
    return {"metric": "all-pairs/s, inbred / ill-conditioned stress", "value": pairs / (t * 1e-3),
            "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
            "higher_is_better": True, "dtype": "f32" if args.precision == "fp32c" else "f64",
            "data": "synthetic",
            "config": {"workload": f"N={n} x M={co.codes.shape[1]}, 128 inbred, 32 identical-inbred pairs, "
                                   "5,000-site low-information block", "pairs": pairs},
            "flagged_cond_gt_1e15": int(np.sum(~(np.log10(np.where(cond > 0, cond, np.nan)) <= 15))),
            "stats": {k: st[k] for k in ("gh_passes", "fp64_pairs", "fp64_passes", "waves", "nonconverged")}}


def run_serving(args, local):
    """A resident 4,096 x 100,000 panel; query batches of 1-64 samples, each with
    its own site mask, arrive as a Poisson stream at 200 requests/s and are
    submitted at their arrival times; latency = completion - arrival."""
    import concurrent.futures as cf
    import kestrel_b200 as kb
    from kestrel_b200 import synth
    panel = synth.config4_panel()
    reqs = synth.config4_requests(panel, args.requests, rate_hz=args.rate)
    warm = synth.config4_requests(panel, 4, seed=7)
    est = kb.Estimator(device=local, precision=args.precision)
    est.panel_load(panel.codes)
    for r in warm:
        est.wait(est.submit(r["codes"], r["site_mask"]))
    n_panel = panel.codes.shape[0]
    done_t = {}
    pool = cf.ThreadPoolExecutor(max_workers=len(reqs))

    def waiter(rid, i):
        est.wait(rid)
        done_t[i] = time.perf_counter()

    futs = []
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        delay = t0 + r["arrival_s"] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        rid = est.submit(r["codes"], r["site_mask"])
        futs.append(pool.submit(waiter, rid, i))
    for f in futs:
        f.result()
    pool.shutdown()
    lat = np.array([(done_t[i] - (t0 + r["arrival_s"])) * 1e3 for i, r in enumerate(reqs)])
    span = max(done_t.values()) - t0
    pairs = sum(r["codes"].shape[0] * n_panel for r in reqs)
    sv = est.serving_stats()
    est.close()
    return {"metric": "serving pairs/s; query p50/p99 ms", "value": pairs / span, "unit": "pairs/s",
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "n_gpus": 1, "requests": len(reqs), "higher_is_better": True,
            "dtype": "f32" if args.precision == "fp32c" else "f64", "data": "synthetic",
            "config": {"workload": f"panel {n_panel} x {panel.codes.shape[1]}, Poisson {args.rate:g} req/s, 1-64 query "
                                   "samples, per-request site mask keeping U(0.6, 1.0) of sites",
                       "pairs": pairs},
            "timing": "host wall clock from the first arrival to the last completion; latency per request "
                      "from its arrival time to the return of its kg_wait",
            "launches": sv["launches"]}


def run_gl_soft(args, local):
    """The GL/PL estimator on soft genotype likelihoods (kg_relatedness_gl): all
    pairs of --samples x --sites, likelihoods with mass off the call (each
    other genotype uniform in [0, 0.05) of the called one's), 2% missing."""
    import torch
    import kestrel_b200 as kb
    from kestrel_b200 import synth
    from oracle import pyoracle
    n_s, m_s = args.samples, args.sites
    co = synth.make_cohort(n_s, m_s, 9, missing=0.02, planted={"parent_offspring": 4, "full_sib": 4},
                           name="gl-soft")
    rng = np.random.default_rng(10)
    c = co.codes                                          # [samples, sites]
    gl = rng.uniform(0.0, 0.05, c.shape + (3,))
    for g in range(3):
        gl[..., g] = np.where(c == g, 1.0, gl[..., g])
    gl[c == synth.MISSING] = np.nan
    pairs = n_s * (n_s + 1) // 2
    est = kb.Estimator(device=local, precision=args.precision)
    est.load_likelihoods(gl)
    for _ in range(max(3, args.warmup)):
        est.relatedness_gl()
    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    clocks.start()
    dev, st = [], None
    for _ in range(max(1, args.steps)):
        est.relatedness_gl()
        st = est.run_stats()
        dev.append(st["device_ms"])
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = float(np.mean(dev))
    peak = ctypes_peak(local)
    achieved = st["flops_fp32"] / (t * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None, "traffic": None, "kernel": "soft_pairs_kernel",
            "peak_source": "kg_fp32_peak (FFMA loop over all SMs, measured in this run)",
            "flops_counted": "FP32 evaluations at 204 FLOP per pair-site (the row from the nine likelihood "
                             "products, d, gradient, 45 Hessian terms, objective; FMA = 2) over the device time "
                             "of the whole call; FP64 re-evaluations excluded",
            "note": "the FP32 likelihoods (12 bytes per sample-site) stay L2-resident at this size"}
    gl_pin = torch.from_numpy(gl).pin_memory().numpy()
    out_pin = torch.empty(pairs * kb.OUTPUT_DTYPE.itemsize, dtype=torch.uint8,
                          pin_memory=True).numpy().view(kb.OUTPUT_DTYPE)
    e2e_ms = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        est.load_likelihoods(gl_pin)
        est.relatedness_gl(out=out_pin)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    te = float(np.mean(e2e_ms))
    est.close()
    cpu = None
    if not args.no_cpu:
        sub = min(n_s, 48)
        t0 = time.perf_counter()
        pyoracle.gl_relatedness(np.ascontiguousarray(gl[:sub].transpose(1, 0, 2)))
        dt = time.perf_counter() - t0
        cpu = {"value": sub * (sub + 1) / 2 / dt, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"all {sub * (sub + 1) // 2} pairs of the first {sub} samples (oracle FP64 GL "
                         f"restatement, OpenMP over {os.cpu_count()} threads, {dt:.1f} s)"}
    return {"metric": "all-pairs/s, GL/PL estimator on soft likelihoods", "value": pairs / (t * 1e-3),
            "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32c" else "f64", "data": "synthetic",
            "config": {"workload": f"all pairs of N={n_s} x M={m_s} soft likelihoods (2% missing)", "pairs": pairs},
            "e2e": {"value": pairs / (te * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": int(gl.nbytes),
                    "d2h_bytes_per_step": int(out_pin.nbytes), "ms_per_step": te},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(st["launches"]),
            "stats": {k: st[k] for k in ("gh_passes", "fp64_passes", "fp64_pairs", "work_units")}}


def run_ml_multi(args, local):
    """The ML estimator with tri- and tetra-allelic sites beside the biallelic
    ones: all pairs of --samples x --sites (the headline cohort) plus
    --multi-sites (default 10,000) tri-/tetra-allelic sites with 2% missing
    calls, device time per step, and the same cohort without them."""
    import torch
    import kestrel_b200 as kb
    from kestrel_b200 import synth
    n_s, m_s = args.samples, args.sites
    nm = args.multi_sites or 10_000
    co = synth.config1(n_samples=n_s, n_sites=m_s)
    mg, mal = synth.make_multiallelic(n_s, nm, 3, missing=0.02)
    pairs = n_s * (n_s - 1) // 2
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    est = kb.Estimator(device=local, precision=args.precision)
    res = {}
    for label, multi in (("with", True), ("without", False)):
        est.load(co.codes)
        if multi:
            est.load_multiallelic(mg, mal)
        for _ in range(max(3, args.warmup)):
            est.relatedness()
        dev, st = [], None
        for _ in range(max(1, args.steps)):
            flush.zero_()
            torch.cuda.synchronize()
            est.relatedness()
            st = est.run_stats()
            dev.append(st["device_ms"])
        res[label] = (float(np.mean(dev)), st)
    est.close()
    t, st = res["with"]
    return {"metric": "all-pairs/s, ML estimator with tri-/tetra-allelic sites", "value": pairs / (t * 1e-3),
            "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t,
            "higher_is_better": True, "dtype": "f32" if args.precision == "fp32c" else "f64", "data": "synthetic",
            "config": {"workload": f"all pairs of N={n_s} x M={m_s} + {nm} tri-/tetra-allelic sites (2% missing)",
                       "pairs": pairs, "l2": "256 MB buffer written between steps"},
            "without_multiallelic": {"value": pairs / (res["without"][0] * 1e-3), "ms_per_step": res["without"][0]},
            "phases_ms": {"admit": st["admit_ms"], "pass_and_multi": st["pass_ms"], "solve": st["solve_ms"]},
            "stats": {k: st[k] for k in ("gh_passes", "fp64_pairs", "waves", "sites_used", "nonconverged")}}


def run_gt_cls(args, local):
    """The reference's default hard-call estimator (-f GT: conditional least
    squares, Brier objective) on all pairs of N=1024 x M=100,000 with every call
    present (the GT reader drops a site with a missing call): one CLS moment
    pass per pair and the simplex QP, through kg_relatedness_gt."""
    import torch
    import kestrel_b200 as kb
    from kestrel_b200 import synth
    from oracle import pyoracle
    n_s, m_s = args.samples, args.sites
    k = min(64, n_s // 16)
    co = synth.make_cohort(n_s, m_s, 1, missing=0.0,
                           planted={"parent_offspring": k, "full_sib": k, "half_sib": k, "first_cousin": k},
                           name="gt-cls")
    codes = co.codes
    pairs = n_s * (n_s - 1) // 2
    mg, mal = synth.make_multiallelic(n_s, args.multi_sites, 2) if args.multi_sites else (None, None)
    est = kb.Estimator(device=local, precision=args.precision)
    est.load(codes)
    if mg is not None:
        est.load_multiallelic(mg, mal)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(max(3, args.warmup)):
        est.relatedness_gt()
    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    clocks.start()
    dev, st = [], None
    for _ in range(max(1, args.steps)):
        flush.zero_()
        torch.cuda.synchronize()
        est.relatedness_gt()
        st = est.run_stats()
        dev.append(st["device_ms"])
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = float(np.mean(dev))
    # end to end: upload from pinned memory, estimate, all rows back, per step
    codes_pin = torch.from_numpy(codes).pin_memory().numpy()
    out_pin = torch.empty(n_s * (n_s + 1) // 2 * kb.OUTPUT_DTYPE.itemsize, dtype=torch.uint8,
                          pin_memory=True).numpy().view(kb.OUTPUT_DTYPE)
    # (on the same context: a second one would find half the memory taken)
    est.load(codes_pin)
    if mg is not None:
        est.load_multiallelic(mg, mal)
    est.relatedness_gt(out=out_pin)
    e2e_ms = []
    for _ in range(max(1, args.steps)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        est.load(codes_pin)
        if mg is not None:
            est.load_multiallelic(mg, mal)
        est.relatedness_gt(out=out_pin)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    te = float(np.mean(e2e_ms))
    # the list-building (admit) kernel dominates: HBM-bound, 4 bytes written per
    # listed pair-site; the moment pass reads them once
    pair_sites = float(st["pair_sites"])
    admit_ms, pass_ms = st["admit_ms"], st["pass_ms"]
    top = "wave_admit_kernel" if admit_ms >= pass_ms else "wave_pass_kernel"
    top_ms = max(admit_ms, pass_ms)
    achieved = 4.0 * pair_sites / (top_ms * 1e-3) / 1e9
    peak = measured_hbm_peak()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if peak else None, "traffic": None, "kernel": top,
            "algorithmic_bytes": 4.0 * pair_sites / max(1, int(st["waves"])),
            "note": "4 bytes per listed pair-site (written by the admit kernel, read once by the moment pass)"}
    cpu = None
    if not args.no_cpu:
        sub = min(n_s, 192)
        t0 = time.perf_counter()
        pyoracle.cls_relatedness(codes[:, :], num_samples=sub,
                                 multi=None if mg is None else (mg, mal, None))
        dt = time.perf_counter() - t0
        cpu = {"value": sub * (sub + 1) / 2 / dt, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"all {sub * (sub + 1) // 2} pairs of the first {sub} samples (oracle FP64 CLS "
                         f"restatement, OpenMP over {os.cpu_count()} threads, {dt:.1f} s)"}
    est.close()
    return {"metric": "all-pairs/s, GT CLS/Brier estimator", "value": pairs / (t * 1e-3), "unit": "pairs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": t,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32c" else "f64", "data": "synthetic",
            "config": {"workload": f"all pairs of N={n_s} x M={m_s}" +
                                   (f" + {args.multi_sites} tri-/tetra-allelic sites" if mg is not None else "") +
                                   ", no missing calls (planted PO/FS/HS/FC)",
                       "pairs": pairs, "l2": "256 MB buffer written between steps"},
            "e2e": {"value": pairs / (te * 1e-3), "unit": "pairs/s",
                    "h2d_bytes_per_step": int(codes.nbytes) + (0 if mg is None else int(mg.nbytes + mal.nbytes)),
                    "d2h_bytes_per_step": int(out_pin.nbytes), "ms_per_step": te},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": int(st["launches"]),
            "phases_ms": {"admit": admit_ms, "pass": pass_ms, "solve": st["solve_ms"]},
            "stats": {k2: st[k2] for k2 in ("gh_passes", "waves", "slots", "nonconverged", "pair_sites")}}


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.workload != "allpairs":
        import torch
        torch.cuda.set_device(local)
        fn = {"batch": run_batch, "inbred": run_inbred, "serving": run_serving, "gt-cls": run_gt_cls,
              "gl-soft": run_gl_soft, "ml-multi": run_ml_multi}[args.workload]
        if rank == 0:
            print(json.dumps(fn(args, local)), flush=True)
        return
    from kestrel_b200 import synth
    cohort = synth.config1(n_samples=args.samples, n_sites=args.sites)
    codes = cohort.codes
    if args.impl == "reference":
        run_reference(args, codes, cohort.planted)
        return
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    import kestrel_b200 as kb
    from kestrel_b200 import _lib
    n, m = codes.shape
    pairs = n * (n - 1) // 2
    est = kb.Estimator(device=local, precision=args.precision)
    est.set_launch(args.slots, args.pass_bps)
    est.load(codes)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        est.relatedness()
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    dev_ms, kern_ms, fl32, phases, stats = [], [], [], [], None
    for _ in range(args.steps):
        flush.zero_()          # evict L2 between steps
        torch.cuda.synchronize()
        rows = est.relatedness()
        stats = est.run_stats()
        dev_ms.append(stats["device_ms"])
        kern_ms.append(stats["pass_ms"])
        fl32.append(stats["flops_fp32"])
        phases.append([stats["admit_ms"], stats["pass_ms"], stats["solve_ms"], stats["pair_kernel_ms"]])
    barrier()
    clk = clocks.stop()
    t_step = max(dev_ms) if dev_ms else float("nan")
    t_mean = float(np.mean(dev_ms))
    t_mean = max_over_ranks(t_mean, pg, f"cuda:{local}")
    value = whole_job_rate(pairs, world, t_mean)
    # ---- end to end through the C ABI from pinned host buffers: every step
    # uploads the genotypes in the VCF reader's packed form (2-bit codes plus
    # the observed mask, kg_load_genotypes_2bit), estimates and copies all rows
    # back (kg_relatedness); the context is made once, as a caller would (the
    # same one: a second context would find half the memory taken by the
    # first one's slots and run with fewer)
    e2e = None
    if not args.no_e2e:
        c2, ob = kb.pack_2bit(codes)
        c2_pin = torch.from_numpy(c2.view(np.int32)).pin_memory().numpy().view(np.uint32)
        ob_pin = torch.from_numpy(ob.view(np.int32)).pin_memory().numpy().view(np.uint32)
        out_pin = torch.empty(n * (n + 1) // 2 * kb.OUTPUT_DTYPE.itemsize, dtype=torch.uint8,
                              pin_memory=True).numpy().view(kb.OUTPUT_DTYPE)
        est.load_packed(c2_pin, ob_pin, m)
        est.relatedness(out=out_pin)         # warm
        e2e_ms = []
        for i in range(max(1, args.steps)):
            flush.zero_()
            barrier()
            t0 = time.perf_counter()
            est.load_packed(c2_pin, ob_pin, m)
            est.relatedness(out=out_pin)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        tm = max_over_ranks(float(np.mean(e2e_ms)), pg, f"cuda:{local}")
        e2e = {"value": whole_job_rate(pairs, world, tm), "unit": "pairs/s",
               "h2d_bytes_per_step": int(c2.nbytes + ob.nbytes), "d2h_bytes_per_step": int(out_pin.nbytes),
               "ms_per_step": tm, "timing": "host wall clock around the synchronous C-ABI calls per step "
                                            "(packed genotypes up from pinned memory, estimate, all rows to "
                                            "pinned memory)"}
    # ---- roofline of the site-pass kernel (FP32 CUDA-core bound; FP64 for the FP64 form)
    peak32 = ctypes_peak(local)
    kms = float(np.mean(kern_ms))
    launches = max(1, int(stats["waves"]))           # one pass launch per wave
    pass_sites = float(stats["work_units"])          # pair-site evaluations of the step
    fp64_form = args.precision == "fp64"
    flops = float(stats["flops_fp64"]) if fp64_form else float(np.mean(fl32))
    peak = (peak32 / 2.0 if peak32 else None) if fp64_form else peak32
    achieved = flops / (kms * 1e-3) / 1e12
    ref_equiv = pass_sites * 156.0 / (kms * 1e-3) / 1e12
    list_bytes = 8.0 if fp64_form else 4.0
    roof = {"bound": "fp64" if fp64_form else "fp32", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
            # DRAM bytes per pair-site-pass from one ncu capture (a 96-sample
            # cohort), times the pair-sites of an average pass launch of this step
            "traffic": (PASS_DRAM_BYTES_PER_SITE * pass_sites / launches) if not fp64_form else None,
            "traffic_unit": "bytes per launch",
            "algorithmic_bytes": list_bytes * pass_sites / launches,
            "hbm_achieved_gbs": list_bytes * pass_sites / (kms * 1e-3) / 1e9,
            "hbm_peak_gbs": measured_hbm_peak(),
            "kernel": "wave_pass_kernel", "kernel_ms": kms, "launches": launches,
            "kernel_timing": "device clock (%globaltimer) from the first block's start to the last warp's end "
                             "of every wave's site-pass launch, summed per step",
            "peak_source": ("half of kg_fp32_peak (B200 FP64 CUDA-core rate)" if fp64_form else
                            "kg_fp32_peak (FFMA loop over all SMs, measured in this run)"),
            "flops_counted": ("executed site arithmetic of the shape-moment passes (FMA = 2, MUFU = 1) "
                              "per shape and pass kind; FP64 re-evaluation passes excluded" if not fp64_form
                              else "executed FP64 site arithmetic of the shape-moment passes (FMA = 2)"),
            "ref_formulation_tflops": ref_equiv,
            "ref_formulation_note": "the same pair-site-passes counted at the reference formulation's "
                                    "136 + 20 FLOP (dense 9 + 45 sums); the shape moments need 19-41"}
    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mean,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32c" else "f64",
            "data": "synthetic",
            "config": workload_config(n, m),
            "precision": args.precision, "parallelism": f"replicas x{world}",
            "e2e": e2e, "roofline": roof, "clocks": clk,
            "gpu_launches": int(stats["launches"]) * args.steps,
            "phases_ms": dict(zip(("admit", "pass", "solve", "waves_total"),
                                  [float(v) for v in np.mean(np.array(phases), axis=0)])),
            "stats": {k: stats[k] for k in ("gh_passes", "fp64_passes", "fp64_pairs", "pair_sites",
                                            "work_units", "shape_sites", "waves", "slots", "nonconverged",
                                            "flops_fp64")}}
    if rank == 0 and world == 1 and args.precision == "fp32c" and not args.no_fp64:
        line["fp64_form"] = measure_fp64_form(est, value)
    if rank == 0 and not args.no_cpu and world == 1:
        cb, sp, sr, fr = cpu_baseline(codes, cohort.planted, args.cpu_seconds, keep_rows=True)
        line["cpu_baseline"] = cb
        line["error_vs_oracle"] = error_vs_oracle(rows, codes, cohort.planted, sp, sr, fr)
    if rank == 0:
        print(json.dumps(line), flush=True)
    est.close()
    if pg:
        pg.destroy_process_group()


def measure_fp64_form(est, fp32c_value, steps=2):
    """The plain FP64 GPU form (every site pass in FP64, IEEE division and the
    library log) on the same loaded cohort, after the FP32C timing: pairs/s
    from the device time of `steps` calls after one warm-up, and the FP32C
    form's speed-up over it."""
    est.set_precision("fp64")
    try:
        est.relatedness()
        dev = []
        for _ in range(steps):
            est.relatedness()
            dev.append(est.run_stats()["device_ms"])
    finally:
        est.set_precision("fp32c")
    t = float(np.mean(dev))
    n = est.n_samples
    v = n * (n - 1) // 2 / (t * 1e-3)
    return {"value": v, "unit": "pairs/s", "ms_per_step": t, "steps": steps,
            "ratio_fp32c_over_fp64": fp32c_value / v,
            "timing": "device time (CUDA events in the library) of kg_relatedness with KG_PREC_FP64"}


# DRAM bytes (read + write) per pair-site-pass of wave_pass_kernel: the ncu
# capture of one launch on a 96-sample x 100,000-site cohort read and wrote
# 1.912 GB over 447,339,158 pair-site-passes.
PASS_DRAM_BYTES_PER_SITE = 4.27


def ctypes_peak(device):
    import ctypes
    from kestrel_b200 import _lib
    v = ctypes.c_double()
    st = _lib.lib().kg_fp32_peak(device, ctypes.byref(v))
    return v.value if st == 0 else None


if __name__ == "__main__":
    main()
