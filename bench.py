"""Benchmark of the subpixel-metrology hot path on B200 (one JSON line on rank 0).

Workload (one step): the 8192 x 8192 uint16 staggered contact-hole page (pitch 24, d 12 +- 5 %,
sigma 1.2, ~116k holes incl. border-clipped), synthetic and seeded: detect_centers with the three
refiners (weighted, logquad, edge_gradmoment) and measure_cds (model background, LM Gaussian-FWHM,
radial-gradient and half-height CDs, summary_only), all through the public API.

  value  cells/s with the page already in HBM (a CUDA tensor passed to the API)
  e2e    cells/s through the same API with a host (NumPy) page: host->device copy of the page and
         device->host copy of the results inside the timed region
  accuracy_vs_oracle
         the GPU pipeline (warm-started and plain) against the FP64 CPU oracle on the CPU-baseline
         crop of the same page: largest centre and CD errors per method, same seeds / statuses
  lm_stage
         the initial-fit stage in three arms: plain LM at the reference's 1e-12 stop rule, plain LM
         at the warm fits' 1e-7 rule (like for like), and patches + MLP + warm-started LM

Cells = Voronoi cells reported and measured by the LM Gaussian method. The page (134 MB) is larger
than the 126 MB L2, so consecutive steps do not run from cache.

``--tiled`` measures the tiled detection instead (one JSON line of its own): detect_centers_tiled
(tile_h 8192, overlap 128, global Otsu) on a 32768 x 32768 uint16 square array (pitch 20, d 10,
~2.7M holes) rendered on the device, with the graph-captured band pipeline and with the eager one.

``--stack`` measures the uneven stack instead (one JSON line of its own): 64 synthetic 4096 x 4096
uint16 images, each with its own pitch U(16, 40) px, hole diameter 0.4-0.6 x pitch, 5 % missing and
2 % merged holes; the initial LM fits of all their cells run in one launch, warm-started (patches,
MLP, LM: `value`) and plain (`plain_lm`), with the warm start's deviation from the plain FP64 fit
per image; `full_measure_cds` then times measure_cds of every image (image by image on the GPU) and
checks each against the FP64 oracle on a 384 x 384 corner.

``--impl reference`` times the CPU path (the oracle restatement of the reference algorithm, NumPy /
SciPy on the host cores) on a crop of the same page; under torchrun only rank 0 runs it.
Multi-GPU: one process per GPU, each measuring its own page (weak scaling, no collective on the
data path); the step time is the max over ranks.
"""

from __future__ import annotations

import argparse
import contextlib
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cells/s on 1 B200 at ≤1e-3 px vs FP64: NN-warm-started LM vs plain LM"
UNIT = "cells/s"
WORKLOAD = "page_staggered_8192x8192_u16_pitch24_d12_3refiners_3cd"
METHODS = ("gaussian", "gradient", "halfmax")
REFINERS = ("weighted", "logquad", "edge_gradmoment")
CD_KW = dict(area_max=400, summary_only=True)
CENTER_KW = dict(threshold="otsu", area_max=400)
# Algorithmic FP64 operations of one k_fit_iteration launch (adds and multiplies, an FMA counted
# as two, exp and rsqrt as one each), counted from the cells' own work in the timed launches:
#   per staged pixel, cleaning (own Gaussian, background, model): FIT_FLOP_CLEAN
#   per staged pixel and LM pass (one pass at the start, one per iteration): model, residual, cost,
#     the six Jacobian entries, 21 J^T J and 6 J^T r accumulations: FIT_FLOP_PASS
#   per LM iteration, the damped 6x6 Cholesky solve, trial step and acceptance: FIT_FLOP_SOLVE
FIT_FLOP_CLEAN = 16.0
FIT_FLOP_PASS = 83.0
FIT_FLOP_SOLVE = 185.0
# DRAM bytes (read + write) per cell of one k_fit_iteration launch and the FP64 instructions it
# issues per cell (dadd + dmul + 2 dfma, exp expanded), constants from one ncu capture of a launch
# on the 4096x4096 page (29,241 cells: 190.3 MB of DRAM traffic, 15.42 GFLOP issued in 1.094 ms),
# not measured in this run; both scale with the cells processed.
FIT_TRAFFIC_PER_CELL = 6508.0
FIT_ISSUED_FLOP_PER_CELL = 5.274e5


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms; started before the warm-up (its
    start-up takes driver locks that would stall the timed steps) and summarised over the samples
    taken between mark_start() and mark_end()."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.window = (None, None)

    def mark_start(self):
        self.window = (time.monotonic(), None)

    def mark_end(self):
        self.window = (self.window[0], time.monotonic())

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append((time.monotonic(), parts))

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        t0, t1 = self.window
        inside = [p for t, p in self.samples if (t0 is None or t >= t0) and (t1 is None or t <= t1)]
        where = "inside the timed region"
        if not inside and t0 is not None:
            # A timed region shorter than the 200 ms sampling period: the samples just before and
            # just after it (the GPU was busy with the warm-up and the end-to-end steps then).
            before = [(t, p) for t, p in self.samples if t < t0]
            after = [(t, p) for t, p in self.samples if t1 is not None and t > t1]
            inside = [q[-1][1] for q in (before, after[:1]) if q]
            where = "adjacent to a timed region shorter than the sampling period"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in inside if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in inside if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in inside for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(inside), "sampled": where}


def make_page(rank: int, size: int = 8192):
    from imageprocessor_new_b200 import synthetic

    return synthetic.page_staggered(seed=rank, shape=(size, size)).image


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    from imageprocessor_new_b200 import _lib, deblend, detect_centers, measure_cds

    rank, world, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    page = make_page(rank, args.page)
    page_d = torch.from_numpy(page).cuda()
    lib = _lib.lib()

    # Dominant-kernel timing: CUDA events around every LM deblending iteration (one k_fit_iteration
    # launch each) on the launching stream, inside the timed region.
    fit_times = []
    fit_cells = []
    fit_work = []  # (iterations, staged pixels) per cell of every timed launch, device tensors
    orig_iteration = deblend.Deblender.iteration

    def timed_iteration(self, params_d, model, bg):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        out = orig_iteration(self, params_d, model, bg)
        e.record()
        fit_times.append((s, e))
        fit_cells.append(self.n)
        fit_work.append((out[3], self.cells.counts))
        return out

    deblend.Deblender.iteration = timed_iteration

    def step(image):
        for refine in REFINERS:
            detect_centers(image, backend="gpu", refine=refine, **CENTER_KW)
        return measure_cds(image, backend="gpu", methods=METHODS, **CD_KW)

    def warm(image, k):
        # As in the timed loop, each step runs while the previous step's results are still held:
        # the results are views of pinned host buffers, so the host allocator reaches its steady
        # state (two sets of download buffers) before the timed steps.
        res = None
        for _ in range(k):
            res = step(image)
        return res

    def run(image, k):
        fit_times.clear()
        fit_cells.clear()
        fit_work.clear()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = lib.spx_launch_count()
        s.record()
        cells = 0
        for _ in range(k):
            res = step(image)
            cells += len(res.seeds_xy)
        e.record()
        torch.cuda.synchronize()
        launches = lib.spx_launch_count() - n0
        ms = s.elapsed_time(e)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        return ms, cells, launches

    # Launch shapes from the autotuner (timed on this page's cells, outside the timed region).
    from imageprocessor_new_b200 import autotune, warmstart

    tuned = autotune.tune(page_d, use_cache=False)["config"] if args.autotune else autotune.current()

    # Variants: the NN-warm-started pipeline (when a trained model is present) and the plain one.

    model_path = Path(args.model) if args.model else warmstart.DEFAULT_MODEL
    net = warmstart.WarmStartNet.load(model_path) if (args.warm_start and model_path.exists()) else None
    timings, results = {}, {}
    for variant in ["plain"] + (["warm"] if net is not None else []):
        warmstart.use(net if variant == "warm" else None)
        headline = variant == ("warm" if net is not None else "plain")
        with (ClockSampler(local) if headline else contextlib.nullcontext()) as clocks:
            warm(page_d, args.warmup)
            if headline:
                clocks.mark_start()
            ms_v, cells_v, launches_v = run(page_d, args.steps)
            if headline:
                clocks.mark_end()
                clock_summary = clocks.summary()
        timings[variant] = (ms_v, cells_v, launches_v)
        if headline:
            ms, cells, launches = ms_v, cells_v, launches_v
            fit_ms = [a.elapsed_time(b) for a, b in fit_times]
            fit_avg_ms = float(np.mean(fit_ms)) if fit_ms else float("nan")
            fit_n = float(np.mean(fit_cells)) if fit_cells else 0.0
            fit_flop = _fit_flops(fit_work)
            # End to end: host page, copies inside the region.
            warm(page, max(2, args.warmup))
            ms_e2e, cells_e2e, _ = run(page, args.steps)
        results[variant] = step(page_d)
    lm_stage = warmstart.compare_on_page(net, page_d) if (net is not None and world == 1) else None
    warmstart.use(None)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    per_step_cells = cells / args.steps
    value = world * per_step_cells / (ms / 1e3 / args.steps)
    e2e = world * (cells_e2e / args.steps) / (ms_e2e / 1e3 / args.steps)
    peaks, which = _peaks()
    d2h = _d2h_bytes(int(per_step_cells))
    # Roofline of the dominant kernel, the LM deblending iteration: FP64-bound (neither a tensor-core
    # contraction nor HBM-bound), so its roofline is the FP64 rate measured here on this GPU, and the
    # achieved rate is the launches' algorithmic FP64 operations over their CUDA-event time. Its
    # HBM view beside it: algorithmic bytes = the cells' pixels read (image 2 B + labels 4 B + model
    # 8 B + background rows 8 B) plus 6 params in / 6 out + status.
    fp64_peak = fp64_peak_tflops()
    fit_tflops = fit_flop / (sum(fit_ms) / 1e3) / 1e12 if fit_ms else None
    px_per_cell = 24 * 24
    bytes_per_cell = px_per_cell * (2 + 4 + 8 + 8) + 13 * 8
    achieved_gbs = fit_n * bytes_per_cell / (fit_avg_ms / 1e3) / 1e9 if fit_ms else None
    mpix = world * args.page * args.page / 1e6 / (ms / 1e3 / args.steps)
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded render + noise)",
        "config": {"workload": _workload(args.page), "image": f"{args.page}x{args.page} uint16",
                   "cells_per_step": per_step_cells,
                   "methods": list(METHODS), "refiners": list(REFINERS),
                   "l2": f"inputs {'larger' if page.nbytes > 126e6 else 'smaller'} than L2 "
                         f"({page.nbytes / 1e6:.0f} MB page)",
                   "warm_start": "plain LM (no network)"},
        "e2e": {"value": round(e2e, 1), "unit": UNIT, "h2d_bytes_per_step": int(page.nbytes) * (len(REFINERS) + 1),
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "fp64", "kernel": "k_fit_iteration<double>", "unit": "TFLOP/s",
                     "achieved": None if fit_tflops is None else round(fit_tflops, 3),
                     "peak": round(fp64_peak, 3),
                     "peak_source": "measured in this run (spx_fp64_fma_rate: independent DFMA chains on "
                                    "every SM, CUDA events)",
                     "frac": None if fit_tflops is None else round(fit_tflops / fp64_peak, 4),
                     "flop_per_launch": round(fit_flop / max(len(fit_ms), 1)),
                     "flop_source": "algorithmic, from the timed launches' per-cell LM iterations and staged "
                                    "pixels (exp and rsqrt one operation each)",
                     "issued_frac": None if not fit_ms else
                     round(FIT_ISSUED_FLOP_PER_CELL * fit_n / (fit_avg_ms / 1e3) / 1e12 / fp64_peak, 4),
                     "issued_source": "FP64 instructions issued per cell (exp expanded) from one ncu capture "
                                      "(4096x4096 page), scaled by cells",
                     "traffic": round(FIT_TRAFFIC_PER_CELL * fit_n / 1e9, 4), "traffic_unit": "GB per launch",
                     "traffic_source": "constant per cell from one ncu capture (4096x4096 page), scaled by cells",
                     "launch_ms": round(fit_avg_ms, 4), "cells_per_launch": fit_n,
                     "hbm": {"achieved": None if achieved_gbs is None else round(achieved_gbs, 1),
                             "peak": peaks.get("hbm_gbs"), "peak_source": which, "unit": "GB/s",
                             "frac": None if achieved_gbs is None else round(achieved_gbs / peaks["hbm_gbs"], 4)}},
        "mpix_per_s": round(mpix, 1),
        "gpu_launches": int(launches),
        "clocks": clock_summary,
    }
    line["config"]["launch_shapes"] = tuned
    if net is not None:
        ms_p, cells_p, _ = timings["plain"]
        line["config"]["warm_start"] = f"MLP 1024-256-256-7 ({model_path.name}), plain-start fallback"
        line["plain_lm"] = {"value": round(world * (cells_p / args.steps) / (ms_p / 1e3 / args.steps), 1),
                            "unit": UNIT, "ms_per_step": round(ms_p / args.steps, 3)}
        line["accuracy_vs_plain"] = _accuracy(results["warm"], results["plain"])
        if lm_stage is not None:
            line["lm_stage"] = {k: (round(v, 6) if isinstance(v, float) else v) for k, v in lm_stage.items()}
    if args.cpu_baseline and world == 1:
        line["cpu_baseline"], oracle_res = cpu_baseline(page, args.cpu_sample)
        crop = np.ascontiguousarray(page[:args.cpu_sample, :args.cpu_sample])
        line["accuracy_vs_oracle"] = {"sample": line["cpu_baseline"]["sample"]}
        for variant in ["plain"] + (["warm"] if net is not None else []):
            warmstart.use(net if variant == "warm" else None)
            line["accuracy_vs_oracle"][variant] = _accuracy_vs_oracle(crop, oracle_res)
        warmstart.use(None)
    print(json.dumps(line), flush=True)


def _accuracy(warm, plain) -> dict:
    """Largest differences of the warm-started pipeline's results from the plain pipeline's (same
    cells): centres and equivalent CDs of every method, in pixels, over cells valid in both."""
    out = {"same_cells": bool(np.array_equal(warm.seeds_xy, plain.seeds_xy))}
    if not out["same_cells"]:
        return out
    for name in METHODS:
        a, b = warm.measurements[name], plain.measurements[name]
        both = a.valid & b.valid
        dc = float(np.abs(a.centers_xy[both] - b.centers_xy[both]).max()) if both.any() else 0.0
        dcd = (float(np.abs(a.metrics["cd_equivalent_px"][both] - b.metrics["cd_equivalent_px"][both]).max())
               if both.any() else 0.0)
        out[name] = {"centre_max_px": dc, "cd_max_px": dcd, "same_validity": float((a.valid == b.valid).mean())}
    return out


def _fit_flops(work) -> float:
    """Algorithmic FP64 operations of the timed k_fit_iteration launches (FIT_FLOP_* per staged
    pixel, per pixel and LM pass, and per iteration), from each launch's per-cell iteration counts
    and staged pixel counts (device tensors, read after the timed region)."""
    total = 0.0
    for iters, pixels in work:
        it = iters.double()
        px = pixels.double()
        total += float((px * (FIT_FLOP_CLEAN + FIT_FLOP_PASS * (it + 1.0))).sum() + FIT_FLOP_SOLVE * it.sum())
    return total


def fp64_peak_tflops(repeats: int = 5) -> float:
    """The device's FP64 rate measured here (spx_fp64_fma_rate: independent FMA chains on every SM,
    CUDA events, best of `repeats`), the denominator of the LM kernel's FP64 roofline."""
    import ctypes

    import torch

    from imageprocessor_new_b200 import _lib

    lib = _lib.lib()
    blocks = 148 * 16
    sink = torch.empty(blocks * 256, dtype=torch.float64, device="cuda")
    flops = ctypes.c_double(0.0)
    stream = torch.cuda.current_stream().cuda_stream
    best = 0.0
    for _ in range(repeats + 1):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        _lib.call("spx_fp64_fma_rate", blocks, 4096, sink.data_ptr(), ctypes.byref(flops), stream)
        e.record()
        torch.cuda.synchronize()
        best = max(best, flops.value / (s.elapsed_time(e) / 1e3) / 1e12)
    return best


def _accuracy_vs_oracle(crop, oracle_res) -> dict:
    """The GPU pipeline on the crop (the three refiners' centres and measure_cds) against the FP64
    CPU oracle's results on the same crop: same seeds and statuses, largest centre / CD errors."""
    from imageprocessor_new_b200 import detect_centers, measure_cds

    centers, cds = oracle_res
    out = {"refiners": {}}
    for refine in REFINERS:
        got = detect_centers(crop, backend="gpu", refine=refine, **CENTER_KW).centers_xy
        want = centers[refine]
        same = got.shape == want.shape
        out["refiners"][refine] = {"same_count": bool(same),
                                   "centre_max_px": float(np.abs(got - want).max(initial=0.0)) if same else None}
    res = measure_cds(crop, backend="gpu", methods=METHODS, area_max=400)
    out["same_seeds"] = bool(np.array_equal(res.seeds_xy, cds["seeds"]))
    out["same_cell_labels"] = bool(np.array_equal(res.cell_labels, cds["cell_labels"]))
    if not out["same_seeds"]:
        return out
    for m in METHODS:
        got, want = res.measurements[m], cds["measurements"][m]
        both = got.valid & (want["status"] == "ok")
        a, b = got.metrics["cd_equivalent_px"][both], want["metrics"]["cd_equivalent_px"][both]
        dc = np.abs(got.centers_xy[both] - want["centers"][both])
        out[m] = {"cells": int(len(got.valid)), "same_status": float((got.status == want["status"]).mean()),
                  "centre_max_px": float(dc.max(initial=0.0)), "cd_max_px": float(np.abs(a - b).max(initial=0.0))}
    worst_c = max([out[m]["centre_max_px"] for m in METHODS] +
                  [r["centre_max_px"] or 0.0 for r in out["refiners"].values()])
    worst_cd = max(out[m]["cd_max_px"] for m in METHODS)
    out["within_1e-3_px_centres"] = bool(worst_c <= 1e-3)
    out["within_2e-3_px_cds"] = bool(worst_cd <= 2e-3)
    return out


def _workload(size: int) -> str:
    return WORKLOAD if size == 8192 else WORKLOAD.replace("8192x8192", f"{size}x{size}")


def _d2h_bytes(cells: int) -> int:
    """Result bytes copied to the host per step: each CD method's output buffer (one copy per method)
    and the three refiners' centre arrays."""
    from imageprocessor_new_b200 import cd

    total = 0
    for method in METHODS:
        b, _ = cd._method_buffers(cells, 128, method, False)
        total += b["_flat"].numel() * 8
    return total + len(REFINERS) * cells * 16


def cpu_baseline(page, size):
    """The oracle (CPU restatement of the reference path) on a crop of the page, all host cores.
    Returns the baseline entry and the oracle's results ({refiner: centres}, measure_cds dict)."""
    from oracle import cd as ocd
    from oracle import centers as oc

    crop = np.ascontiguousarray(page[:size, :size])
    t0 = time.perf_counter()
    centers = {}
    for refine in REFINERS:
        centers[refine] = oc.detect_centers(crop, threshold="otsu", refine_method=refine, area_max=400)
    res = ocd.measure_cds(crop, methods=METHODS, area_max=400)
    dt = time.perf_counter() - t0
    n = len(res["seeds"])
    return ({"value": round(n / dt, 2), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
             "sample": f"{size}x{size} crop of the page ({n} cells), same step", "seconds": round(dt, 2)},
            (centers, res))


def reference_arm(args):
    rank, world, _ = _dist()
    if rank != 0:
        return
    page = make_page(0)
    size = args.cpu_sample
    for _ in range(max(0, min(args.warmup, 1))):
        pass
    vals, secs, cells = [], [], 0
    for _ in range(args.steps):
        r, _ = cpu_baseline(page, size)
        vals.append(r["value"])
        secs.append(r["seconds"])
    value = float(np.median(vals))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * float(np.mean(secs)), 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded render + noise)",
            "config": {"workload": WORKLOAD, "sample": f"{size}x{size} crop"}, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{size}x{size} crop of the page, same step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def tiled_arm(args):
    """detect_centers_tiled on the 32768 x 32768 page: centres/s with band graphs and eagerly."""
    import torch

    from imageprocessor_new_b200 import synthetic, tiled

    torch.cuda.set_device(0)
    page_d, truth = synthetic.page_large_device(0, args.tiled_size)
    torch.cuda.synchronize()
    kw = dict(threshold="otsu", invert=False, area_min=1, area_max=400, pad=3, refine="auto", connectivity=8,
              small_feature_max=12.0, tile_h=8192, overlap=128, threshold_mode="global", otsu_downsample=4,
              thr_scale=0.8, dedupe_eps=1.5, device=0)
    out = {}
    for name, graphs in (("graphs", True), ("eager", False)):
        for _ in range(max(1, args.warmup)):
            res = tiled.detect_tiled(page_d, use_graphs=graphs, **kw)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(args.steps):
            res = tiled.detect_tiled(page_d, use_graphs=graphs, **kw)
        e.record()
        torch.cuda.synchronize()
        out[name] = (s.elapsed_time(e) / args.steps, len(res.centers_xy), res)
    ms, n, res = out["graphs"]
    px = args.tiled_size ** 2
    cpu = tiled_cpu_baseline(page_d, res, args) if args.cpu_baseline else None
    print(json.dumps({
        "metric": "centres/s, detect_centers_tiled", "value": round(n / (ms / 1e3), 1), "unit": "centres/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "mpix_per_s": round(px / 1e6 / (ms / 1e3), 1), "centres": n, "true_holes": int(len(truth)),
        "band_graphs": bool(res.meta["band_graphs"]),
        "eager": {"ms_per_step": round(out["eager"][0], 3),
                  "value": round(out["eager"][1] / (out["eager"][0] / 1e3), 1)},
        "graphs_equal_eager": bool(np.array_equal(res.centers_xy, out["eager"][2].centers_xy)),
        "dtype": "u16 in, f64 centres", "data": "synthetic (rendered on the device)",
        "config": {"workload": f"page_square_{args.tiled_size}x{args.tiled_size}_u16_pitch20_d10_tiled",
                   "tile_h": 8192, "overlap": 128, "threshold": "otsu (global, img[::4, ::4] x 0.8)",
                   "refine": "auto"},
        "cpu_baseline": cpu}), flush=True)


def tiled_cpu_baseline(page_d, res, args, strip_rows: int = 512) -> dict:
    """The tiled page's CPU cost by the oracle (the reference algorithm on the host cores), from
    bounded samples: the global Otsu of img[::4, ::4]; the per-band detection timed on one strip of
    `strip_rows` rows (fixed threshold, refine="auto") and scaled by the rows the bands cover
    (overlaps counted twice); the reference's O(N^2) dedupe timed on 1/64 of the page's centres and
    extrapolated by (64)^2. Centres/s = the page's centres / the extrapolated total."""
    from imageprocessor_new_b200 import shard
    from oracle import centers as oc
    from oracle import segment as osg

    size = int(page_d.shape[0])
    t0 = time.perf_counter()
    sub = page_d[::4, ::4].cpu().numpy()
    pre = osg.otsu_threshold(np.ascontiguousarray(sub)) * 0.8
    t_otsu = time.perf_counter() - t0
    y0 = size // 2
    strip = page_d[y0:y0 + strip_rows].cpu().numpy()
    t0 = time.perf_counter()
    oc.detect_centers(strip, threshold="otsu", area_max=400, refine_method="auto", fixed_threshold=pre)
    t_strip = time.perf_counter() - t0
    rows = sum(b.y1 - b.y0 for b in shard.band_plan(size, 8192, 128))
    t_bands = t_strip * rows / strip_rows
    pts = res.centers_xy[:: 64]
    t0 = time.perf_counter()
    oc.dedupe_pairwise(pts, 1.5)
    t_dd = time.perf_counter() - t0
    t_total = t_otsu + t_bands + t_dd * 64 ** 2
    return {"value": round(len(res.centers_xy) / t_total, 2), "unit": "centres/s", "cores": os.cpu_count(),
            "kind": "port", "sample": (f"global Otsu of img[::4, ::4]; one {strip_rows}-row strip of detection "
                                       f"scaled by the {rows} band rows; O(N^2) dedupe on 1/64 of the centres "
                                       "extrapolated by 64^2"),
            "seconds": {"otsu": round(t_otsu, 2), "strip": round(t_strip, 2), "bands_extrapolated": round(t_bands, 1),
                        "dedupe_1_64": round(t_dd, 2), "dedupe_extrapolated": round(t_dd * 64 ** 2, 1),
                        "page_extrapolated": round(t_total, 1)}}


def stack_arm(args):
    """All cells of the uneven stack in one initial-fit launch: cells/s warm-started and plain."""
    import torch

    from imageprocessor_new_b200 import _lib
    from imageprocessor_new_b200 import stack as st
    from imageprocessor_new_b200 import warmstart as ws

    torch.cuda.set_device(0)
    s = st.synth_stack(args.stack_images, args.stack_size, seed=0)
    sc = st.stack_cells(s)
    net = ws.WarmStartNet.load(args.model) if args.model else ws.WarmStartNet.load()
    arms = {"warm": lambda: st.initial_fits(s, sc, net=net), "plain": lambda: st.initial_fits(s, sc)}
    ms = {k: 0.0 for k in arms}
    res = {}
    with ClockSampler(0) as clocks:
        for _ in range(max(3, args.warmup)):
            for fn in arms.values():
                fn()
        torch.cuda.synchronize()
        clocks.mark_start()
        n0 = _lib.lib().spx_launch_count()
        for _ in range(args.steps):
            for k, fn in arms.items():
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                res[k] = fn()
                b.record()
                torch.cuda.synchronize()
                ms[k] += a.elapsed_time(b) / args.steps
        launches = _lib.lib().spx_launch_count() - n0
        clocks.mark_end()
    net.check_errors()
    (pw, sw, iw, _, fw), (pp, sp, ip, _, _) = ([t.cpu().numpy() for t in res[k]] for k in ("warm", "plain"))
    per_image = []
    for i in range(sc.images):
        sl = sc.image_of(i)
        ok = (sw[sl] == 0) & (sp[sl] == 0)
        dev = np.abs(pw[sl][ok, 1:3] - pp[sl][ok, 1:3]).max(initial=0.0)
        per_image.append({"cells": int(sl.stop - sl.start), "centre_dev_max_px": float(dev),
                          "same_status": float((sw[sl] == sp[sl]).mean()) if sl.stop > sl.start else 1.0,
                          "plain_iterations_mean": round(float(ip[sl].mean()), 3) if sl.stop > sl.start else 0.0,
                          "warm_iterations_mean": round(float(iw[sl].mean()), 3) if sl.stop > sl.start else 0.0})
    n = sc.n
    full = stack_full_pipeline(s)
    cpu = stack_cpu_baseline(s, args) if args.cpu_baseline else None
    print(json.dumps({
        "metric": METRIC, "value": round(n / (ms["warm"] / 1e3), 1), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": round(ms["warm"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (rendered on the device)",
        "config": {"workload": f"stack_{args.stack_images}x{args.stack_size}x{args.stack_size}_u16_uneven",
                   "cells": n, "images": sc.images, "launch": "one initial-fit launch over all cells of the stack",
                   "l2": f"inputs larger than L2 ({s.numel() * 2 / 1e9:.1f} GB stack)"},
        "plain_lm": {"value": round(n / (ms["plain"] / 1e3), 1), "unit": UNIT, "ms_per_step": round(ms["plain"], 3)},
        "speedup": round(ms["plain"] / ms["warm"], 3),
        "gpu_launches": int(launches),
        "fallback_fraction": float(fw.mean()),
        "centre_dev_max_px": max(p["centre_dev_max_px"] for p in per_image),
        "within_1e-3_px": bool(all(p["centre_dev_max_px"] <= 1e-3 for p in per_image)),
        "per_image": per_image, "clocks": clocks.summary(), "cpu_baseline": cpu,
        "full_measure_cds": full}), flush=True)


STACK_CD_KW = dict(area_min=10, area_max=2000, pad=3)


def _stack_oracle_worker(crop):
    """One pool worker: the oracle's measure_cds of one image crop (no GPU here)."""
    from oracle import cd as ocd

    return ocd.measure_cds(crop, methods=METHODS, **STACK_CD_KW)


def stack_full_pipeline(stack_d, crop: int = 384) -> dict:
    """measure_cds (the bench's methods, summary_only) of every image of the stack, one after another
    on this GPU, timed with CUDA events (the images already in HBM); and per image the GPU pipeline
    against the FP64 oracle on a crop x crop corner (a spawn pool on the host cores): largest centre
    and CD differences per method over the cells both report."""
    import multiprocessing as mp

    import torch

    from imageprocessor_new_b200 import measure_cds

    n_img = int(stack_d.shape[0])
    measure_cds(stack_d[0], backend="gpu", methods=METHODS, summary_only=True, **STACK_CD_KW)
    torch.cuda.synchronize()
    per_image, cells, total = [], 0, 0.0
    for i in range(n_img):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        res = measure_cds(stack_d[i], backend="gpu", methods=METHODS, summary_only=True, **STACK_CD_KW)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        total += ms
        cells += len(res.seeds_xy)
        per_image.append({"cells": int(len(res.seeds_xy)), "ms": round(ms, 3)})
    crops = [np.ascontiguousarray(stack_d[i, :crop, :crop].cpu().numpy()) for i in range(n_img)]
    with mp.get_context("spawn").Pool(max(1, min(n_img, os.cpu_count() or 1))) as pool:
        oracle = pool.map(_stack_oracle_worker, crops)
    worst_c = worst_cd = 0.0
    same = True
    for i, (c, ref) in enumerate(zip(crops, oracle)):
        got = measure_cds(c, backend="gpu", methods=METHODS, **STACK_CD_KW)
        same = same and np.array_equal(got.seeds_xy, ref["seeds"])
        err_c = err_cd = 0.0
        if np.array_equal(got.seeds_xy, ref["seeds"]):
            for m in METHODS:
                g, r = got.measurements[m], ref["measurements"][m]
                both = (g.status == "ok") & (r["status"] == "ok")
                if both.any():
                    err_c = max(err_c, float(np.abs(g.centers_xy[both] - r["centers"][both]).max()))
                    err_cd = max(err_cd, float(np.abs(g.metrics["cd_equivalent_px"][both]
                                                      - r["metrics"]["cd_equivalent_px"][both]).max()))
        per_image[i].update(oracle_crop_cells=int(len(ref["seeds"])), centre_max_px=err_c, cd_max_px=err_cd)
        worst_c, worst_cd = max(worst_c, err_c), max(worst_cd, err_cd)
    return {"value": round(cells / (total / 1e3), 1), "unit": UNIT, "ms_total": round(total, 2), "cells": cells,
            "how": "measure_cds (gaussian, gradient, halfmax; summary_only) image by image on one GPU",
            "accuracy_vs_oracle": {"sample": f"{crop}x{crop} corner of every image", "same_seeds": same,
                                   "centre_max_px": worst_c, "cd_max_px": worst_cd},
            "per_image": per_image}


def _stack_cpu_worker(crop):
    """One pool worker: the oracle's initial fits of one image crop's cells, timed (no GPU here)."""
    import time as _time

    from oracle import cd as ocd
    from oracle import deblend as odb

    seeds, masks, origins = ocd.threshold_cells(crop, area_min=10, area_max=2000, pad=3)
    t0 = _time.perf_counter()
    odb.initial_fits(crop, seeds, masks, origins)
    return len(seeds), _time.perf_counter() - t0


def stack_cpu_baseline(stack_d, args, crop: int = 768) -> dict:
    """The stack's initial fits on the host cores by the oracle (the reference's NumPy LM), as the
    reference's batch pipeline runs them: a process pool of min(64, cores) workers, one image each,
    on a bounded sample (a crop x crop corner of the first `workers` images). cells/s = cells fitted
    / the pool's wall time for the fits (the slowest worker bounds it)."""
    import multiprocessing as mp

    workers = max(1, min(64, os.cpu_count() or 1, int(stack_d.shape[0])))
    crops = [np.ascontiguousarray(stack_d[i, :crop, :crop].cpu().numpy()) for i in range(workers)]
    with mp.get_context("spawn").Pool(workers) as pool:
        out = pool.map(_stack_cpu_worker, crops)
    cells = sum(c for c, _ in out)
    wall = max(t for _, t in out)
    return {"value": round(cells / wall, 2), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "workers": workers, "sample": f"{crop}x{crop} corner of each of {workers} images, one per worker",
            "cells": cells, "seconds": round(wall, 2)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=("gpu", "reference"))
    ap.add_argument("--cpu-sample", type=int, default=768)
    ap.add_argument("--page", type=int, default=8192, help="page side in pixels (8192 = the benchmark page)")
    ap.add_argument("--model", default=None, help="warm-start MLP (default: the packaged model)")
    ap.add_argument("--no-warm-start", dest="warm_start", action="store_false")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--tiled", action="store_true", help="measure detect_centers_tiled on the 32768^2 page instead")
    ap.add_argument("--tiled-size", type=int, default=32768)
    ap.add_argument("--stack", action="store_true", help="measure the uneven 64 x 4096^2 stack in one launch instead")
    ap.add_argument("--stack-images", type=int, default=64)
    ap.add_argument("--stack-size", type=int, default=4096)
    args = ap.parse_args()
    if args.tiled:
        tiled_arm(args)
    elif args.stack:
        stack_arm(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
