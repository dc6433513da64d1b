"""Benchmark of the TLS search on B200: light curves per second.

Default workload (one step = one full search of one light curve, as
``gtls(t, y, dy).power()`` runs it: main pass over every trial period, SDE
spectra, FP64 re-search of the 200 candidates and 5 harmonics, best-period
finish):

  long-baseline FP64 search -- 70,000 samples at 29.4-min cadence over
  ~1,470 d with 17 gaps, per-sample sigma U(50, 500) ppm + AR(1) red noise,
  one 490 ppm transit at P = 289.9 d; Ofir grid 0.5-735 d at oversampling 3
  (187,850 periods), 50 durations.  Seeded synthetic data.

``value`` is device-timed with the inputs resident in HBM; ``e2e`` times the
public API from host arrays (host->device copies and result readback inside
the timed region).  Under torchrun every rank searches its own light curve
(independent replicas, no collective in the data path; weak scaling) and
``value`` is the total over ranks.  ``--impl reference`` times the
reference's own kernel code compiled for the host CPU (oracle/_ref, all
cores) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "light curves/s (long-baseline TLS search, 70k samples, 187,850 periods x 50 durations)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"],
                    help="main-pass precision (default: fp32 for cfg4, fp64 otherwise)")
    ap.add_argument("--workload", default="cfg2", choices=["cfg2", "cfg1", "cfg3", "cfg4", "cfg5"])
    ap.add_argument("--curves", type=int, default=32,
                    help="cfg4: curves per step (every 4096/curves-th curve of the 4,096-curve set)")
    ap.add_argument("--no-per-curve", action="store_true", help="cfg4: skip the per-curve FP64 comparison")
    ap.add_argument("--accuracy", action="store_true",
                    help="cfg4: only the agreement of the batched FP32 search with the plain FP64 per-curve "
                         "search over the sample (one pass each), no timing steps")
    ap.add_argument("--once", action="store_true",
                    help="cfg4: one end-to-end gtls_batch call over the sample (e.g. --curves 4096: the whole set), "
                         "after a small warm-up call; wall clock, no timing steps")
    ap.add_argument("--tuning", default=None,
                    help="fixed launch shapes 'tile_cap_fp32,tile_cap_fp64,bucket_shift[,records_global]' instead of "
                         "autotuning "
                         "(profiling runs: ncu slows untimed launches, which would skew the tuner)")
    ap.add_argument("--chunk-mb", type=int, default=0,
                    help="per-chunk scratch budget of the searches in MiB (default: the library's 8 GiB)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched FP32 vs per-curve FP64 comparison on a sample of the 4,096-curve set")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the leg that times the reference's own kernels on the same GPU")
    ap.add_argument("--max-periods", type=int, default=0,
                    help="profiling only: keep this many periods spread over the grid (a smaller case of the "
                         "same kernels); the line then describes that case")
    return ap.parse_args()


def traffic_per_period(precision, workload):
    """DRAM bytes per period of the chi2 kernel from a recorded ncu capture
    (profiles/chi2_kernel_traffic.txt: lines 'workload precision bytes_per_period'), or None."""
    path = os.path.join(ROOT, "profiles", "chi2_kernel_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) == 3 and parts[0] == workload and parts[1] == precision:
                return float(parts[2])
    except OSError:
        pass
    return None


def durations_step_for(periods, n, want):
    """duration_grid_step giving exactly ``want`` durations."""
    from gtls_b200.grid import duration_grid_step_for
    return duration_grid_step_for(periods, 1 / n, want)


def workload(name, rank=0):
    from gtls_b200 import synthetic, validate as V
    if name == "cfg2":
        t, y, dy, truth = synthetic.light_curve_cfg2(seed=rank)
        kw = dict(period_min=0.5, period_max=735.0, oversampling_factor=3)
        n_dur = 50
        desc = "cfg2: 70,000 samples, 29.4-min cadence, ~1,470 d, 17 gaps; Ofir 0.5-735 d osf 3; 50 durations"
    else:
        t, y, dy, truth = synthetic.light_curve_cfg1(seed=rank)
        kw = dict(period_min=0.5, period_max=13.7, oversampling_factor=3)
        n_dur = None
        desc = "cfg1: 19,728 samples, 2-min cadence, 27.4 d + 1 d gap; Ofir 0.5-13.7 d osf 3; default durations"
    t, y, dy = V.validate_inputs(t, y, dy)
    return t, y, dy, truth, kw, n_dur, desc


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region.  The raw
    samples go to GTLS_CLOCKS_DIR (default: the system temporary directory);
    the JSON line carries their summary."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        out = os.environ.get("GTLS_CLOCKS_DIR")
        self.keep = bool(out)
        self.path = os.path.join(out or tempfile.gettempdir(), "clocks_%d.csv" % os.getpid())
        self._summary = None

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if self._summary is None:
            self._summary = self._read()
            if not self.keep and os.path.exists(self.path):
                os.remove(self.path)
        return self._summary

    def _read(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference(t, y, dy, periods, kw, step, batch_hint, budget_s=15.0, seed=0):
    """Time the reference's kernels (compiled for the CPU, all host cores) on a
    sample of the workload and extrapolate to one full search."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_replay as RR
    import tls_oracle as O
    from gtls_b200 import grid as G, template
    if not RR.available("r64_skip8"):
        return None
    durs = G.duration_grid(periods, shortest=1 / len(t), log_step=step)
    mw = int(np.max(durs) * len(y))
    mw += mw % 2
    ov, lc = template.get_cache(durs, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    widths, os_, _, tm, maxd = template.device_templates(lc, ov)
    rb = RR.RefKernelBackend("r64", 8)
    rng = np.random.default_rng(seed)
    span = t.max() - t.min()
    wmin, wmax = O.duration_ranges(periods, span, len(t))
    masks = O.duration_masks(wmin, wmax, widths)
    unions = O.batch_unions(masks, batch_hint)
    main_t, main_n, all_t, all_n = 0.0, 0, 0.0, 0
    t_begin = time.time()
    order = rng.permutation(len(periods))
    i = 0
    while time.time() - t_begin < budget_s * 0.75 and i < len(order):
        p = order[i]
        sel = unions[p // batch_hint]
        a = time.time()
        rb.main_pass(t, y, dy, periods[p], widths[sel], tm[sel], os_[sel], maxd, 1e-5, 8)
        main_t += time.time() - a
        main_n += 1
        i += 1
    while time.time() - t_begin < budget_s and all_n < 3:
        p = order[(i + all_n) % len(order)]
        sel = unions[p // batch_hint]
        a = time.time()
        rb.noskip_pass(t, y, dy, periods[p], widths[sel], tm[sel], os_[sel], maxd, 1e-5)
        all_t += time.time() - a
        all_n += 1
    per_main = main_t / max(main_n, 1)
    per_all = all_t / max(all_n, 1) if all_n else per_main * 8
    total = per_main * len(periods) + per_all * 206
    return dict(value=1.0 / total, unit="light curves/s", cores=os.cpu_count(), kind="reference",
                sample="%d main-pass periods + %d all-starts periods of the workload through the reference's "
                       "kernels compiled for the CPU (oracle/_ref, OpenMP, %d threads), extrapolated to %d + 206 "
                       "periods" % (main_n, all_n, os.cpu_count(), len(periods)),
                seconds_per_curve=total)


def pipe_object(timings, chi2_ms, precision):
    """FMA-pipe figures of the main-pass chi2 kernel: 2 FLOP per multiply-add,
    against the nominal FP64 (64 FMA/clk/SM) or FP32 (128) peak at 1.965 GHz.
    ``dense``: every evaluated (start, template sample), whether or not the
    start's window passes the depth test; ``active``: the starts that pass it,
    the only sums that enter the result (the reference's kernel runs its
    in-transit loop for these alone, GPUFun.py:409-424); ``issued``: what the
    kernel executed (register groups of consecutive starts covering the
    passing ones, padded template blocks)."""
    peak = 148 * (64 if precision == "fp64" else 128) * 2 * 1.965e9 / 1e12
    sec = chi2_ms * 1e-3
    out = {"unit": "TFLOP/s", "fp_pipe": "fp64" if precision == "fp64" else "fp32", "nominal_peak": peak,
           "flops": "2 per (start, template sample) for B and for C"}
    for key, name in (("chi2_fma", "dense"), ("chi2_active_fma", "active"), ("chi2_issued_fma", "issued")):
        f = 2.0 * statistics.mean(tm[key] for tm in timings)
        out[name + "_flops_per_step"] = f
        out[name + "_tflops"] = f / sec / 1e12
        out[name + "_frac"] = f / sec / 1e12 / peak
    out["achieved"] = out["issued_tflops"]
    out["frac"] = out["issued_frac"]
    return out


def ref_gpu_leg(cur, t, y, dy, lc, ov, periods, batch, ours_main_s, device, n_sample=6):
    """The reference's own kernels on the same GPU: GPUFun.cu compiled for
    sm_100a (oracle/_ref/libgpufun_ref_sm100.so), launched in the order of its
    type-consistent caller (_worker.py, FP32 flux/weights/sums, torch playing
    cupy's argsort/cumsum/argmin).  A stratified sample of its batches of
    ``batch`` periods is timed (wall clock per batch: the reference reads the
    batch's duration union back to the host every batch) and the main pass is
    extrapolated to all batches.  The sampled periods are also searched here
    in FP64 over the same batches, to compare chi2 minima and locations."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu as RG
    import torch
    from gtls_b200 import _lib
    if not RG.available():
        return None
    rg = RG.RefGpuMainPass(t, y, dy, lc, ov, 1e-5, device)
    rg.prepare(periods, batch)
    nb = rg.n_batches
    pick = np.unique(np.linspace(0, nb - 1, min(n_sample, nb)).astype(int))
    rg.run_batch(int(pick[-1]))   # warm-up: module load, allocations
    torch.cuda.synchronize()
    times, same, total, rel = [], 0, 0, []
    for b in pick:
        torch.cuda.synchronize()
        a = time.perf_counter()
        out = rg.run_batch(int(b))
        torch.cuda.synchronize()
        times.append(time.perf_counter() - a)
        if out is None:
            continue
        v, loc = out
        s0, s1 = int(b) * batch, min((int(b) + 1) * batch, len(periods))
        c, l = cur.search(periods[s0:s1], 1e-5, 8, batch, _lib.GTLS_PASS_MAIN, "fp64", want_loc=True)
        v = v.double().cpu().numpy()
        c = c.cpu().numpy()
        same += int(np.sum(loc.cpu().numpy() == l.cpu().numpy()))
        total += s1 - s0
        rel.append(float(np.max(np.abs(v / c - 1))))
    main_s = float(np.mean(times)) * nb
    del rg
    torch.cuda.empty_cache()
    return {"what": "the reference's kernels (GPUFun.cu, SKIP_POINT 8) compiled for sm_100a and launched as its "
                    "type-consistent caller _worker.py does (R32: FP64 times and phases, FP32 flux, weights and "
                    "sums); torch plays cupy's argsort, cumsum, argmin and logical_or on the same stream; main "
                    "pass only",
            "batches": int(nb), "batch_periods": int(batch), "sampled_batches": [int(b) for b in pick],
            "sampled_batch_s": times, "main_pass_s_extrapolated": main_s, "ours_main_pass_s": ours_main_s,
            "main_pass_speedup": main_s / ours_main_s,
            "r32_vs_ours_fp64": {"periods": total, "same_argmin_location": same / max(total, 1),
                                 "max_rel_chi2_difference": max(rel) if rel else None}}


def batched_headline(device, n_curves=16):
    """The metric's comparison on a sample of the 4,096-curve batched set
    (every 4096/n_curves-th curve): one gtls_batch(...).power() call in the
    FP32-compensated form against gtls(...).power(precision="fp64") per curve
    with the same duration-union batch sizes, both end to end from host
    arrays (wall clock, after one untimed call of each), with the agreement
    of best period index and SDE; the sample's share of the set's work gives
    the extrapolated time of all 4,096 curves."""
    import torch
    from gtls_b200 import gtls, synthetic
    from gtls_b200.batch import gtls_batch, prepare_curve
    from gtls_b200.validate import validate_args
    import types
    specs, idx, total_work = cfg4_sample(n_curves)
    curves = [synthetic.light_curve_cfg4(specs, int(i))[:2] for i in idx]
    opts = types.SimpleNamespace()
    validate_args(opts, dict(use_threads=1, GPUDeviceID=device))
    work = float(sum(len(c[0]) * len(prepare_curve(c[0], c[1], None, opts, device=device,
                                                   templates="device")["periods"]) for c in curves))
    kw = dict(use_threads=1, GPUDeviceID=device, keep_spectra=False)
    out = gtls_batch(curves).power(precision="fp32", **kw)
    torch.cuda.synchronize()
    a = time.perf_counter()
    out = gtls_batch(curves).power(precision="fp32", **kw)
    torch.cuda.synchronize()
    b_s = time.perf_counter() - a
    S = [int(o.batch_periods) for o in out]
    gtls(curves[0][0], curves[0][1], verbose=False).power(precision="fp64", use_threads=1, GPUDeviceID=device,
                                                         batch_periods=S[0])
    torch.cuda.synchronize()
    a = time.perf_counter()
    r64 = [gtls(t, y, verbose=False).power(precision="fp64", use_threads=1, GPUDeviceID=device, batch_periods=s)
           for (t, y), s in zip(curves, S)]
    torch.cuda.synchronize()
    p_s = time.perf_counter() - a
    same = [o.period_index == r.diagnostics["period_index"] for o, r in zip(out, r64)]
    sde = [abs(o.SDE / r.SDE - 1) for o, r in zip(out, r64)]
    return {"what": "batched FP32-compensated search (one gtls_batch call) vs plain FP64 per-curve searches "
                    "(gtls(...).power(precision='fp64') each, same duration-union batch sizes) on every %d-th curve "
                    "of the 4,096-curve set, end to end from host arrays, wall clock" % (4096 // n_curves),
            "curves": len(idx), "work_fraction_of_4096_set": work / total_work,
            "batched_fp32_curves_per_s": len(idx) / b_s, "per_curve_fp64_curves_per_s": len(idx) / p_s,
            "speedup": p_s / b_s, "best_index_agreement": float(np.mean(same)), "sde_max_rel_diff": float(max(sde)),
            "full_set_seconds_batched_estimate": b_s * total_work / work,
            "full_set_seconds_per_curve_fp64_estimate": p_s * total_work / work}


def bench_refine(args):
    """Adjoint refinement workload: 1,024 curves x 20,000 samples, 6 parameters
    each; one step = 50 batched Adam iterations (model chi2 forward + adjoint)."""
    import torch
    from gtls_b200 import _lib, refine, synthetic
    curves, truth, start, scales = synthetic.refinement_set(n_curves=1024, n=20000, seed=0)
    t, y, w, off = refine.pack_curves(curves, "cuda")
    p0 = torch.from_numpy(start).cuda()
    sc = torch.from_numpy(scales).cuda()
    for _ in range(args.warmup):
        refine.refine(p0, sc, t, y, w, off, steps=50)
    torch.cuda.synchronize()
    launches0 = _lib.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        out, chi, better = refine.refine(p0, sc, t, y, w, off, steps=50)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (_lib.launch_count() - launches0) // args.steps
    # end to end from host arrays
    torch.cuda.synchronize()
    a = time.perf_counter()
    t2, y2, w2, off2 = refine.pack_curves(curves, "cuda")
    o2, c2, b2 = refine.refine(torch.from_numpy(start).cuda(), torch.from_numpy(scales).cuda(), t2, y2, w2, off2,
                               steps=50)
    res = o2.cpu().numpy()
    torch.cuda.synchronize()
    e2e_ms = 1000 * (time.perf_counter() - a)
    samples = int(off[-1].item())
    chi_start = refine.model_chi2_function().apply(p0, t, y, w, off)
    gain = float(torch.median(chi_start - chi).item())
    line = {"metric": "light curves/s (adjoint refinement, 50 Adam steps, 1,024 x 20,000 samples)",
            "value": 1024 * 1000.0 / ms, "unit": "light curves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cfg5: 1,024 curves x 20,000 samples, (P,T0,D,depth,u1,u2), 50 Adam steps",
                       "samples": samples},
            "e2e": {"value": 1024 * 1000.0 / e2e_ms, "unit": "light curves/s",
                    "h2d_bytes_per_step": int(samples * 24 + 1025 * 8 + 2 * 1024 * 48),
                    "d2h_bytes_per_step": 1024 * 48, "ms_per_step": e2e_ms},
            "gpu_launches": int(launches),
            "result": {"improved_fraction": float(better.float().mean()), "median_chi2_decrease": gain}}
    print(json.dumps(line))
    return 0


CFG4_METRIC = ("light curves/s (batched TLS search of the 4,096-curve synthetic survey set: 5k-70k samples, "
               "27-1,470 d, per-curve Ofir grids and duration grids)")


def fixed_or_tuned(args, tune_fn, device):
    """Launch shapes for the run: ``--tuning`` if given, else chosen by timing
    on the workload's own data (untimed, before the warm-up).  Sets them on
    the device's context and returns them."""
    from gtls_b200 import _lib
    if args.tuning:
        vals = [int(v) for v in args.tuning.split(",")]
        c32, c64, shift = vals[:3]
        rg = vals[3] if len(vals) > 3 else 0
        _lib.set_tuning(tile_cap_fp32=c32, tile_cap_fp64=c64, bucket_shift=shift, records_global=rg, device=device)
        return _lib.get_tuning(device)
    return tune_fn()


def cfg4_sample(n_curves):
    """Every (4096 / n_curves)-th curve of the 4,096-curve set, and the set's
    total work (sum over curves of samples x trial periods)."""
    from gtls_b200 import grid as G, synthetic
    specs = synthetic.batch_cfg4_specs()
    stride = max(1, 4096 // n_curves)
    idx = np.arange(0, 4096, stride)[:n_curves]
    npts = np.array([G.ofir_coefficients(1.0, 1.0, s)[2] for s in specs["span"]])
    return specs, idx, float(np.sum(specs["n"] * npts))


def cpu_reference_work(t, y, dy, budget_s, seed=0):
    """Seconds of the reference's CPU kernels per (sample x period) of work,
    measured on one curve of the set (main pass of a random sample of its
    periods, plus the all-starts re-search share of one search)."""
    from gtls_b200 import grid as G
    a3, c, npts, _ = G.ofir_coefficients(1.0, 1.0, t.max() - t.min(), 3, 2)
    X = np.arange(npts) + 1.0
    periods = np.sort(1 / (a3 * X + c) ** 3 / 86400)
    r = cpu_reference(t, y, dy, periods, dict(oversampling_factor=3), 1.1, max(1, len(periods) // 30),
                      budget_s=budget_s, seed=seed)
    if r is None:
        return None, None
    return r["seconds_per_curve"] / (len(t) * len(periods)), r


def cfg4_accuracy(args, curves, idx, specs, device):
    """Agreement of the batched FP32-compensated search with the plain FP64
    per-curve search on the same curves: best period index, best duration
    (width), SDE, depth and T0."""
    import types
    import torch
    from gtls_b200 import core, gtls
    from gtls_b200.batch import gtls_batch, prepare_curve
    from gtls_b200.validate import validate_args
    # the reference sizes its duration-union batches from the free GPU memory
    # (core.py:620-628), which differs between one batched call and many
    # single-curve calls; both sides get the sizes of the same free-memory figure
    free0 = torch.cuda.mem_get_info(device)[0]
    opts = types.SimpleNamespace()
    validate_args(opts, dict(use_threads=1, GPUDeviceID=device))
    S = []
    for (t, y) in curves:
        p = prepare_curve(t, y, None, opts, device=device)
        S.append(core.reference_batch_size(len(p["periods"]), len(p["t"]), p["maxd"], len(p["widths"]), free0))
    a = time.perf_counter()
    rb = gtls_batch(curves).power(precision=args.precision, use_threads=1, GPUDeviceID=device, keep_spectra=False,
                                  batch_periods=np.array(S))
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - a
    a = time.perf_counter()
    r64 = [gtls(t, y, verbose=False).power(precision="fp64", use_threads=1, GPUDeviceID=device, batch_periods=int(s))
           for (t, y), s in zip(curves, S)]
    torch.cuda.synchronize()
    t_64 = time.perf_counter() - a
    same_p = np.array([x.period == y.period for x, y in zip(rb, r64)])
    same_w = np.array([x.width == y.durationPoints for x, y in zip(rb, r64)])
    rel = lambda u, v: abs(u - v) / max(abs(v), 1e-300)
    sde = np.array([rel(x.SDE, y.SDE) for x, y in zip(rb, r64)])
    dep = np.array([rel(x.depth, y.depth) for x, y in zip(rb, r64)])
    t0 = np.array([abs(x.T0 - y.T0) for x, y in zip(rb, r64)])
    line = {"metric": "agreement of the batched FP32-compensated search with the plain FP64 per-curve search",
            "config": {"workload": "cfg4: every %d-th of the 4,096 seeded synthetic curves" % (4096 // len(idx)),
                       "curves": len(idx), "precision": args.precision},
            "best_period_index_agreement": float(same_p.mean()), "disagreeing_curves": [int(i) for i in idx[~same_p]],
            "best_duration_agreement": float(same_w.mean()),
            "SDE_max_rel_diff": float(sde.max()), "SDE_median_rel_diff": float(np.median(sde)),
            "depth_max_rel_diff_same_index": float(dep[same_p].max()) if same_p.any() else None,
            "T0_max_abs_diff_days_same_index": float(t0[same_p].max()) if same_p.any() else None,
            "seconds": {"batched": t_batch, "per_curve_fp64": t_64},
            "recovered_1pct": int(sum(abs(r.period - specs["period"][i]) < 0.01 * specs["period"][i]
                                      for r, i in zip(rb, idx) if specs["has_transit"][i])),
            "with_transit": int(sum(bool(specs["has_transit"][i]) for i in idx))}
    print(json.dumps(line))
    return 0


def cfg4_once(args, curves, idx, specs, total_work, device):
    """One end-to-end batched search of the whole sample (the 4,096-curve set
    with --curves 4096), timed by wall clock around the public API call from
    host arrays, after a warm-up call on 8 curves of it."""
    import torch
    from gtls_b200 import _lib, grid as G
    from gtls_b200.batch import gtls_batch
    gtls_batch(curves[:8]).power(precision=args.precision, use_threads=1, GPUDeviceID=device, keep_spectra=False)
    torch.cuda.synchronize()
    tm = _lib.Timing()
    launches0 = _lib.launch_count(device)
    a = time.perf_counter()
    phases = {}
    with Clocks(device) as clk:
        res = gtls_batch(curves).power(precision=args.precision, use_threads=1, GPUDeviceID=device,
                                       keep_spectra=False, timing=tm, phases=phases)
        torch.cuda.synchronize()
    sec = time.perf_counter() - a
    work = float(sum(len(c[0]) * G.ofir_coefficients(1.0, 1.0, np.ptp(c[0]))[2] for c in curves))
    line = {"metric": CFG4_METRIC + " -- one end-to-end call", "value": len(idx) / sec, "unit": "light curves/s",
            "n_gpus": 1, "seconds": sec, "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "cfg4: %d of the 4,096 seeded synthetic curves in one gtls_batch call" % len(idx),
                       "curves": len(idx), "work_fraction_of_4096_set": work / total_work,
                       "precision": args.precision, "timing": "wall clock around gtls_batch(curves).power() from "
                                                             "host arrays (grids, templates, uploads included)"},
            "main_pass_stages_ms": {k: tm.as_dict()[k] for k in ("setup_ms", "prepare_ms", "chi2_ms", "finish_ms")},
            "phases_s": phases,
            "gpu_launches": int(_lib.launch_count(device) - launches0),
            "result": {"recovered_1pct": int(sum(abs(r.period - specs["period"][i]) < 0.01 * specs["period"][i]
                                                 for r, i in zip(res, idx) if specs["has_transit"][i])),
                       "with_transit": int(sum(bool(specs["has_transit"][i]) for i in idx))},
            "clocks": clk.summary()}
    print(json.dumps(line))
    return 0


def bench_batch(args):
    """cfg4: batched search of a fixed sample of the 4,096-curve set per step."""
    import types
    import torch
    from gtls_b200 import _lib, batch, gtls, synthetic
    from gtls_b200.validate import validate_args
    specs, idx, total_work = cfg4_sample(args.curves)
    curves = [synthetic.light_curve_cfg4(specs, int(i))[:2] for i in idx]
    desc = ("cfg4: every %d-th of the 4,096 seeded synthetic curves (%d per step); FP32-compensated main pass, "
            "FP64 re-search of 200 candidates + 5 harmonics per curve" % (4096 // args.curves, len(idx)))
    if args.impl == "reference":
        # seconds per unit work of the reference's CPU kernels, measured on the
        # sample curve of median work, times the sample's work
        from gtls_b200 import validate as V
        works = [len(c[0]) for c in curves]
        steps = []
        res = None
        sample_work = None
        for i in range(args.warmup + args.steps):
            j = int(np.argsort(works)[len(works) // 2])
            t, y, dy = V.validate_inputs(curves[j][0], curves[j][1], None)
            spw, r = cpu_reference_work(t, y, dy, budget_s=3.0 if i < args.warmup else 10.0, seed=i)
            if spw is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
                return 0
            if sample_work is None:
                from gtls_b200 import grid as G
                sample_work = sum(len(c[0]) * G.ofir_coefficients(1.0, 1.0, np.ptp(c[0]))[2] for c in curves)
            if i >= args.warmup:
                steps.append(spw * sample_work)
                res = r
        sec = statistics.median(steps)
        v = len(idx) / sec
        line = {"metric": CFG4_METRIC, "value": v, "unit": "light curves/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
                "config": {"workload": desc, "curves": len(idx)},
                "cpu_baseline": dict(value=v, unit="light curves/s", cores=res["cores"], kind="reference",
                                     sample=res["sample"] + "; per-(sample x period) cost scaled to the step's "
                                                          "%.3g sample-periods" % sample_work),
                "e2e": {"value": v, "unit": "light curves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    device = torch.cuda.current_device()
    if args.accuracy:
        return cfg4_accuracy(args, curves, idx, specs, device)
    if args.once:
        return cfg4_once(args, curves, idx, specs, total_work, device)
    opts = types.SimpleNamespace()
    validate_args(opts, dict(precision=args.precision, use_threads=1, GPUDeviceID=device))
    prepared = [batch.prepare_curve(t, y, None, opts, device=device, templates="device") for (t, y) in curves]
    cs = batch.CurveSetOnDevice(prepared, device=device)
    from gtls_b200 import tune
    tuning = fixed_or_tuned(args, lambda: tune.tune_curve_set(cs, args.precision), device)
    work = float(sum(len(p["t"]) * len(p["periods"]) for p in prepared))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=cs.dev)
    for _ in range(args.warmup):
        batch.search_on_device(cs, opts, keep_spectra=False)
    torch.cuda.synchronize()
    launches0 = _lib.launch_count(device)
    step_ms, timings = [], []
    with Clocks(device) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            tm = _lib.Timing()
            e0.record()
            out = batch.search_on_device(cs, opts, keep_spectra=False, timing=tm)
            e1.record()
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            timings.append(tm.as_dict())
    launches = (_lib.launch_count(device) - launches0) // args.steps
    ms = statistics.mean(step_ms)

    # end to end through the public batched API from host arrays
    _lib.TRANSFER.update(h2d=0, d2h=0)
    torch.cuda.synchronize()
    a = time.perf_counter()
    res = batch.gtls_batch(curves).power(precision=args.precision, use_threads=1, GPUDeviceID=device,
                                         keep_spectra=False)
    torch.cuda.synchronize()
    e2e_ms = 1000.0 * (time.perf_counter() - a)
    h2d, d2h = _lib.TRANSFER["h2d"], _lib.TRANSFER["d2h"]

    chi2_ms = statistics.mean(t["chi2_ms"] for t in timings)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm_peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        hbm_peak, peak_src = 6650.0, "fallback"
    achieved = 24.0 * work / (chi2_ms * 1e-3) / 1e9
    chunks = timings[0]["chunks"]
    line = {
        "metric": CFG4_METRIC, "value": len(idx) * 1000.0 / ms, "unit": "light curves/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "fp32" else "f64",
        "data": "synthetic",
        "config": {"workload": desc, "curves": len(idx), "sample_periods": work,
                   "work_fraction_of_4096_set": work / total_work,
                   "full_set_seconds_estimate": ms * 1e-3 * total_work / work,
                   "l2": "flushed (256 MB write) before every timed step; per-chunk scratch > L2",
                   "precision": args.precision, "tuning": tuning},
        "e2e": {"value": len(idx) * 1000.0 / e2e_ms, "unit": "light curves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "chi2_kernel", "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None, "peak_source": peak_src,
                     "launches_per_step": chunks, "avg_launch_ms": chi2_ms / max(chunks, 1),
                     "algorithmic_bytes": "24*N per (curve, period): t, y, w in FP64"},
        "pipe": pipe_object(timings, chi2_ms, args.precision),
        "stages_ms": {k: statistics.mean(t[k] for t in timings) for k in
                      ("setup_ms", "prepare_ms", "chi2_ms", "finish_ms")},
    }
    truth = [(specs["period"][i], bool(specs["has_transit"][i])) for i in idx]
    starts = statistics.mean(t["chi2_starts"] for t in timings)
    line["trial_evaluations"] = {
        "what": "(period, duration, start) chi2 evaluations of the main pass per step (the re-searches come on top)",
        "per_step": starts, "per_s_device": starts / (ms * 1e-3), "per_s_main_pass_kernel": starts / (chi2_ms * 1e-3)}
    line["result"] = {"recovered_1pct": int(sum(abs(r.period - p) < 0.01 * p for r, (p, h) in zip(out, truth) if h)),
                      "with_transit": int(sum(h for _, h in truth))}
    if not args.no_per_curve:
        # the plain FP64 per-curve form on the same curves: one gtls().power() each
        torch.cuda.synchronize()
        a = time.perf_counter()
        # same duration-union batch sizes as the batched run (the reference's
        # free-memory formula gives different ones at different times)
        ref64 = [gtls(t, y, verbose=False).power(precision="fp64", use_threads=1, GPUDeviceID=device,
                                                 batch_periods=int(o.batch_periods))
                 for (t, y), o in zip(curves, out)]
        torch.cuda.synchronize()
        pc_ms = 1000.0 * (time.perf_counter() - a)
        same = [int(np.argmin(np.abs(p["periods"] - r.period))) == o.period_index
                for p, r, o in zip(prepared, ref64, out)]
        sde_rel = [abs(o.SDE - r.SDE) / abs(r.SDE) for r, o in zip(ref64, out)]
        line["per_curve_fp64"] = {"value": len(idx) * 1000.0 / pc_ms, "unit": "light curves/s",
                                  "ms": pc_ms, "speedup_of_batched_e2e": pc_ms / e2e_ms,
                                  "best_index_agreement": float(np.mean(same)),
                                  "sde_max_rel_diff": float(np.max(sde_rel)),
                                  "note": "gtls(t, y).power(precision='fp64') per curve with the batched run's "
                                          "batch sizes, host arrays, wall clock"}
    line["clocks"] = clk.summary()
    if not args.no_cpu_baseline:
        from gtls_b200 import validate as V
        j = int(np.argsort([len(c[0]) for c in curves])[len(curves) // 2])
        t, y, dy = V.validate_inputs(curves[j][0], curves[j][1], None)
        spw, r = cpu_reference_work(t, y, dy, budget_s=15.0)
        if spw is not None:
            line["cpu_baseline"] = dict(value=len(idx) / (spw * work), unit="light curves/s", cores=r["cores"],
                                        kind="reference",
                                        sample=r["sample"] + "; per-(sample x period) cost scaled to the step's "
                                                             "%.3g sample-periods" % work)
    print(json.dumps(line))
    return 0


def bench_cfg3(args):
    """cfg3: the mixed-precision form over 64 seeded cfg1-shaped curves.

    Every curve is searched with the FP32-compensated main pass (precision
    "fp32": FP32 chi2 and template sums, float-float prefix sums, FP64 fold,
    FP64 re-search of the 200 candidates and 5 harmonics) and with the plain
    FP64 form, whose chi2 matches the FP64 oracle within 1e-9 relative (the
    GPU parity tests).  Reports throughput of both and the FP32 form's error
    against the FP64 one."""
    import torch
    from gtls_b200 import _lib, gtls, synthetic
    from gtls_b200.batch import gtls_batch
    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "unavailable": "cfg3 is an accuracy report of this implementation's "
                                                              "two precisions; the reference has one (FP32) form"}))
        return 0
    device = torch.cuda.current_device()
    curves = [synthetic.light_curve_cfg3(s) for s in range(64)]
    kw = dict(period_min=0.5, period_max=13.7, oversampling_factor=3, use_threads=1, GPUDeviceID=device)
    for prec in ("fp32", "fp64"):
        gtls(curves[0][0], curves[0][1], curves[0][2], verbose=False).power(precision=prec, **kw)
    res, ms = {}, {}
    launches0 = _lib.launch_count(device)
    with Clocks(device) as clk:
        for prec in ("fp32", "fp64"):
            torch.cuda.synchronize()
            a = time.perf_counter()
            res[prec] = [gtls(t, y, dy, verbose=False).power(precision=prec, **kw) for (t, y, dy, _) in curves]
            torch.cuda.synchronize()
            ms[prec] = 1000.0 * (time.perf_counter() - a)
        torch.cuda.synchronize()
        a = time.perf_counter()
        rb = gtls_batch([(t, y, dy) for (t, y, dy, _) in curves]).power(precision="fp32", **kw)
        torch.cuda.synchronize()
        ms["batched_fp32"] = 1000.0 * (time.perf_counter() - a)
    launches = _lib.launch_count(device) - launches0
    r32, r64 = res["fp32"], res["fp64"]
    idx = [int(np.argmin(np.abs(np.asarray(r.periods) - r.period))) for r in r64]
    same_p = [a.period == b.period for a, b in zip(r32, r64)]
    same_w = [a.durationPoints == b.durationPoints for a, b in zip(r32, r64)]
    same_b = [rb_.period == b.period for rb_, b in zip(rb, r64)]
    rel = lambda a, b: abs(a - b) / max(abs(b), 1e-300)
    spec = []
    for a, b in zip(r32, r64):
        c32, c64 = a.diagnostics["chi2_main"], b.diagnostics["chi2_main"]
        ok = np.isfinite(c64) & np.isfinite(c32)
        spec.append(float(np.max(np.abs(c32[ok] - c64[ok]) / np.abs(c64[ok]))))
    # against the FP64 oracle (tests/golden/cfg3_oracle.npz, made by
    # tests/golden/make_cfg3_oracle.py from the reference's kernels built for the CPU)
    vs_oracle = None
    fx_path = os.path.join(ROOT, "tests", "golden", "cfg3_oracle.npz")
    if os.path.exists(fx_path):
        fx = np.load(fx_path)
        k = min(int(fx["n_seeds"]), len(curves))
        forms = {"fp32_per_curve": [(r.diagnostics["period_index"], r.durationPoints, r.SDE, r.depth, r.T0,
                                     np.ma.getdata(r.chi2)) for r in r32],
                 "fp64_per_curve": [(r.diagnostics["period_index"], r.durationPoints, r.SDE, r.depth, r.T0,
                                     np.ma.getdata(r.chi2)) for r in r64],
                 "batched_fp32": [(r.period_index, r.width, r.SDE, r.depth, r.T0, np.ma.getdata(r.chi2)) for r in rb]}
        vs_oracle = {"seeds": k, "what": "FP64 oracle (reference kernels built for the CPU, R64) on the same grids"}
        for name, vals in forms.items():
            sc = [fx["seed%d_scalars" % s] for s in range(k)]
            same = [int(v[0]) == int(o[0]) for v, o in zip(vals, sc)]
            same_w = [int(v[1]) == int(o[2]) for v, o in zip(vals, sc)]
            spec = []
            for v, s in zip(vals, range(k)):
                o = fx["seed%d_chi2" % s].astype(np.float64)
                ok = np.isfinite(o) & np.isfinite(v[5])
                spec.append(float(np.max(np.abs(v[5][ok] / o[ok] - 1))) if np.any(ok) else 0.0)
            vs_oracle[name] = {"best_period_index_agreement": float(np.mean(same)),
                               "best_duration_agreement": float(np.mean(same_w)),
                               "SDE_max_rel_err": float(max(rel(v[2], o[3]) for v, o in zip(vals, sc))),
                               "depth_max_rel_err": float(max(rel(v[3], o[4]) for v, o in zip(vals, sc))),
                               "T0_max_abs_err_days": float(max(abs(v[4] - o[5]) for v, o in zip(vals, sc))),
                               "chi2_spectrum_max_rel_err": float(max(spec)),
                               "note": "chi2 spectrum against the oracle's stored in float32 (6e-8)"}
    acc = {
        "curves": len(curves),
        "best_period_index_agreement": float(np.mean(same_p)),
        "best_duration_index_agreement": float(np.mean(same_w)),
        "batched_fp32_period_agreement": float(np.mean(same_b)),
        "depth_max_rel_err": float(max(rel(a.depth, b.depth) for a, b in zip(r32, r64))),
        "T0_max_abs_err_days": float(max(abs(a.T0 - b.T0) for a, b in zip(r32, r64))),
        "SDE_max_rel_err": float(max(rel(a.SDE, b.SDE) for a, b in zip(r32, r64))),
        "chi2_spectrum_max_rel_err": float(max(spec)),
        "chi2_spectrum_median_of_max_rel_err": float(np.median(spec)),
        "reference_of_errors": "the plain FP64 form, itself within 1e-9 relative of the FP64 oracle",
    }
    n_periods = int(np.mean([len(r.periods) for r in r64]))
    line = {"metric": "light curves/s (cfg3: 64 seeded cfg1-shaped curves, FP32-compensated form, per-curve calls)",
            "value": 64 * 1000.0 / ms["fp32"], "unit": "light curves/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": ms["fp32"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "cfg3: 64 seeds of 19,728 samples over 27.4 d, depth log-U(100, 2000) ppm, "
                                   "P log-U(1, 500) d; Ofir 0.5-13.7 d osf 3 (~%d periods)" % n_periods,
                       "timing": "wall clock around the public API from host arrays (every step is end to end)"},
            "e2e": {"value": 64 * 1000.0 / ms["fp32"], "unit": "light curves/s", "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": None, "ms_per_step": ms["fp32"]},
            "fp64_per_curve": {"value": 64 * 1000.0 / ms["fp64"], "ms": ms["fp64"]},
            "batched_fp32": {"value": 64 * 1000.0 / ms["batched_fp32"], "ms": ms["batched_fp32"]},
            "gpu_launches": int(launches), "accuracy": acc, "accuracy_vs_fp64_oracle": vs_oracle,
            "clocks": clk.summary()}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.precision is None:
        args.precision = "fp32" if args.workload == "cfg4" else "fp64"
    if args.chunk_mb and args.impl == "ours":
        from gtls_b200 import _lib
        import torch
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        _lib.set_chunk_budget(args.chunk_mb << 20, device=torch.cuda.current_device())
    if args.workload == "cfg5":
        return bench_refine(args)
    if args.workload == "cfg3":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        return bench_cfg3(args)
    if args.workload == "cfg4":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        return bench_batch(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        from gtls_b200 import grid as G
        t, y, dy, truth, kw, n_dur, desc = workload(args.workload)
        a3, c, npts, _ = G.ofir_coefficients(1.0, 1.0, t.max() - t.min(), kw["oversampling_factor"], 2)
        X = np.arange(npts) + 1.0
        periods = 1 / (a3 * X + c) ** 3 / 86400
        periods = np.sort(periods[(periods > kw["period_min"]) & (periods <= kw["period_max"])])
        step = durations_step_for(periods, len(t), n_dur) if n_dur else 1.1
        steps = []
        res = None
        for i in range(args.warmup + args.steps):
            r = cpu_reference(t, y, dy, periods, kw, step, max(1, len(periods) // 30),
                              budget_s=4.0 if i < args.warmup else 12.0, seed=i)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
                return 0
            if i >= args.warmup:
                steps.append(r["seconds_per_curve"])
                res = r
        v = 1.0 / statistics.median(steps)
        line = {"metric": METRIC, "value": v, "unit": "light curves/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * statistics.median(steps),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": desc, "periods": len(periods), "durations": n_dur},
                "cpu_baseline": dict(value=v, unit="light curves/s", cores=res["cores"], kind="reference",
                                     sample=res["sample"]),
                "e2e": {"value": v, "unit": "light curves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    import torch.distributed as dist
    from gtls_b200 import _lib, core, grid as G, gtls
    from gtls_b200.template import get_cache

    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    device = torch.cuda.current_device()
    t, y, dy, truth, kw, n_dur, desc = workload(args.workload, rank)
    periods = np.sort(G.period_grid(1.0, 1.0, t.max() - t.min(), kw["period_min"], kw["period_max"],
                                    kw["oversampling_factor"], 2, device=device, ascending=True))
    step = durations_step_for(periods, len(t), n_dur) if n_dur else 1.1
    if args.max_periods:
        periods = periods[np.linspace(0, len(periods) - 1, args.max_periods).astype(int)]
        desc += " [profiling subset: %d periods]" % len(periods)
    durations = G.duration_grid(periods, shortest=1 / len(t), log_step=step)
    mw = int(np.max(durations) * len(y))
    mw += mw % 2
    ov, lc = get_cache(durations, mw, 12.9, 0.03, 23.1, 89.21, 0, 90, [0.4804, 0.1867], "quadratic")
    cur = core.CurveOnDevice(t, y, dy, lc, ov, device=device)
    periods_dev = torch.from_numpy(periods).to(cur.dev)
    free = torch.cuda.mem_get_info(device)[0]
    batch = core.reference_batch_size(len(periods), cur.n, cur.maxd, len(cur.widths), free)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=cur.dev)  # > 126 MB L2
    from gtls_b200 import tune
    tuning = fixed_or_tuned(args, lambda: tune.tune_curve(cur, periods, args.precision), device)

    def one_step(timing=None, phases=None):
        return core.run_search(cur, periods, periods_dev, t, y, dy, 1e-5, 0.125, kw["oversampling_factor"],
                               precision=args.precision, batch_periods=batch, timing=timing, phases=phases)

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches0 = _lib.launch_count(device)
    timings = []
    step_ms = []
    with Clocks(device) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            tm = _lib.Timing()
            e0.record()
            out = one_step(tm)
            e1.record()
            torch.cuda.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            timings.append(tm.as_dict())
    launches = _lib.launch_count(device) - launches0
    # where one search's time goes: one more (untimed) step with a device
    # synchronisation at each phase boundary
    phases = {}
    one_step(phases=phases)
    total_ms = sum(step_ms)
    if world > 1:
        tt = torch.tensor([total_ms], dtype=torch.float64, device=cur.dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms_per_step = total_ms / args.steps
    value = world * 1000.0 / ms_per_step

    # end to end through the public API from host arrays
    model = gtls(t, y, dy, verbose=False)
    api_kw = dict(period_min=kw["period_min"], period_max=kw["period_max"], batch_periods=batch,
                  duration_grid_step=step, oversampling_factor=kw["oversampling_factor"], precision=args.precision,
                  GPUDeviceID=device)
    if args.max_periods:
        api_kw = dict(periods=periods, batch_periods=batch, duration_grid_step=step,
                      oversampling_factor=kw["oversampling_factor"], precision=args.precision, GPUDeviceID=device)
    model.power(**api_kw)
    torch.cuda.synchronize()
    core.TRANSFER.update(h2d=0, d2h=0)
    e2e_ms = []
    for _ in range(max(1, args.steps // 2)):
        torch.cuda.synchronize()
        a = time.perf_counter()
        model = gtls(t, y, dy, verbose=False)
        model.power(**api_kw)
        torch.cuda.synchronize()
        e2e_ms.append(1000.0 * (time.perf_counter() - a))
    h2d = core.TRANSFER["h2d"] // len(e2e_ms)
    d2h = core.TRANSFER["d2h"] // len(e2e_ms)
    e2e_ms_step = sum(e2e_ms) / len(e2e_ms)
    if world > 1:
        tt = torch.tensor([e2e_ms_step], dtype=torch.float64, device=cur.dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms_step = float(tt.item())

    # roofline of the dominant kernel (chi2), from the library's CUDA events
    chi2_ms = statistics.mean(tm["chi2_ms"] for tm in timings)
    chunks = timings[0]["chunks"]
    n = len(t)
    bytes_per_period = 24 * n   # t, y, w in FP64 per (curve, period)
    achieved_gbs = bytes_per_period * len(periods) / (chi2_ms * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm_peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        hbm_peak, peak_src = 6650.0, "fallback"
    tpp = traffic_per_period(args.precision, args.workload)
    chunk_periods = len(periods) / max(chunks, 1)
    line = {
        "metric": METRIC, "value": value, "unit": "light curves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64", "data": "synthetic",
        "config": {"workload": desc, "periods": len(periods), "durations": len(cur.widths), "samples": n,
                   "batch_periods": batch, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "flushed (256 MB write) before every timed step; per-period scratch > L2",
                   "precision": args.precision, "tuning": tuning},
        "e2e": {"value": world * 1000.0 / e2e_ms_step, "unit": "light curves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms_step},
        "gpu_launches": int(launches // args.steps),
        "roofline": {"bound": "hbm", "kernel": "chi2_kernel", "achieved": achieved_gbs, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved_gbs / hbm_peak,
                     "traffic": (tpp * chunk_periods if tpp else None),
                     "traffic_unit": "bytes per launch (ncu dram read+write per period x periods per launch)",
                     "peak_source": peak_src, "launches_per_step": chunks,
                     "avg_launch_ms": chi2_ms / max(chunks, 1),
                     "algorithmic_bytes": "24*N per (curve, period): t, y, w in FP64",
                     "algorithmic_bytes_per_launch": bytes_per_period * chunk_periods},
        "pipe": pipe_object(timings, chi2_ms, args.precision),
        "stages_ms": {k: statistics.mean(tm[k] for tm in timings) for k in
                      ("setup_ms", "prepare_ms", "chi2_ms", "finish_ms")},
        "phases_ms": {"what": "one extra untimed search, wall clock per phase with a device synchronisation at "
                              "each boundary", **{k: 1000.0 * v for k, v in phases.items()}},
        "result": {"period": float(out[1]), "true_period": truth["period"], "SDE": float(out[7])},
        "trial_evaluations": {
            "what": "(period, duration, start) chi2 evaluations of the main pass per step (the re-searches come on top)",
            "per_step": statistics.mean(tm["chi2_starts"] for tm in timings),
            "per_s_device": statistics.mean(tm["chi2_starts"] for tm in timings) / (ms_per_step * 1e-3),
            "per_s_main_pass_kernel": statistics.mean(tm["chi2_starts"] for tm in timings) / (chi2_ms * 1e-3)},
    }
    if rank == 0:
        line["clocks"] = clk.summary()
        if not args.no_batched and world == 1:
            line["batched"] = batched_headline(device)
        if not args.no_ref_gpu and world == 1:
            main_s = sum(statistics.mean(tm[k] for tm in timings)
                         for k in ("setup_ms", "prepare_ms", "chi2_ms", "finish_ms")) / 1000.0
            rgl = ref_gpu_leg(cur, t, y, dy, lc, ov, periods, batch, main_s, device)
            if rgl is not None:
                line["ref_gpu"] = rgl
        if not args.no_cpu_baseline:
            cb = cpu_reference(t, y, dy, periods, kw, step, batch)
            if cb is not None:
                cb.pop("seconds_per_curve")
                line["cpu_baseline"] = cb
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
