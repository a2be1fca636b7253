"""Autotuner of the launch shapes (no reference counterpart).

The knobs (``spx_tune_set``): warps per block and persistent blocks per SM of the LM fit kernels,
the model-render tile, and how the radial profiles read their spline windows (one ray per thread,
the window cached in registers or read at every sample). None of them changes a result -- the fits take cells from a
device work queue and every cell's arithmetic is the same whatever shape runs it; the render sums
each pixel's Gaussians in cell order in every tile shape; the ray mappings evaluate the same
samples with the same arithmetic and rules -- so the tuner only times them. It times each
candidate with CUDA events on the caller's own data (one initial fit, one deblending iteration and
one render of a page's cells), one knob at a time in the order below, and keeps the fastest. A
choice is cached per device name and workload size class in a JSON file (``SPX_TUNE_CACHE``, or
``autotune.json`` beside this module when unset) and applied with ``apply``.
"""

from __future__ import annotations

import ctypes
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _device as dev
from . import _lib

KNOBS = {
    "fit_warps": (2, 4, 8),
    "fit_blocks_per_sm": (4, 8, 16),
    "render_tile": (16, 32, 64),
    "radial_rays": (0, 2),
}


def get(knob: str) -> int:
    v = ctypes.c_int(0)
    _lib.call("spx_tune_get", knob.encode(), ctypes.byref(v))
    return v.value


def set(knob: str, value: int) -> None:  # noqa: A001 - mirrors the C entry point
    _lib.call("spx_tune_set", knob.encode(), int(value))


def current() -> dict:
    return {k: get(k) for k in KNOBS}


def apply(config: dict) -> None:
    for k, v in config.items():
        set(k, v)


def _cache_path() -> Path:
    return Path(os.environ.get("SPX_TUNE_CACHE", Path(__file__).resolve().parent / "autotune.json"))


def _key(n_cells: int) -> str:
    """Device name and the workload's size class (cells to the nearest power of two)."""
    name = torch.cuda.get_device_name()
    return f"{name}|cells~2^{int(round(np.log2(max(n_cells, 1))))}"


def _time(fn, repeats: int) -> float:
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(repeats):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / repeats


def tune(page_d: torch.Tensor, *, sign: float = 1.0, repeats: int = 3, use_cache: bool = True, log=None) -> dict:
    """Picks the knobs for a page (device image) and applies them; returns the chosen config with
    the timings that decided it."""
    from .deblend import Deblender
    from .warmstart import page_cells

    cells = page_cells(page_d)
    key = _key(cells.n)
    path = _cache_path()
    cache = {}
    if use_cache and path.exists():
        cache = json.loads(path.read_text())
        if key in cache:
            apply(cache[key]["config"])
            return cache[key]
    dbl = Deblender(page_d, sign, cells)
    params, status, _ = dbl.initial(dbl.max_iter)
    model = dbl.render(params)
    bg, _ = dbl.background_of(model, dbl.stats(params, status))

    h, w = dbl.shape
    c = dbl.cells
    cleaned = dev.empty((max(c.n, 1), c.hm, c.wm), torch.float64)
    if c.n:
        _lib.call("spx_clean_cells", dbl.img.data_ptr(), dbl.dtype, dbl.sign, h, w, c.voronoi.data_ptr(),
                  c.boxes.data_ptr(), params.data_ptr(), max(dbl.radius_cap, 2), bg.struct(), model.data_ptr(), None,
                  c.n, c.hm, c.wm, cleaned.data_ptr(), dev.stream_ptr())
    from .cd import _method_buffers

    hb, hs = _method_buffers(c.n, 128, "halfmax", False)
    gb, gs = _method_buffers(c.n, 128, "gradient", False)
    rws = dev.workspace(_lib.size("spx_radial_workspace_bytes", c.hm, c.wm, 0))

    def workload():
        dbl.initial(dbl.max_iter)
        dbl.iteration(params, model, bg)
        dbl.render(params)
        if c.n:
            _lib.call("spx_radial_cd", cleaned.data_ptr(), c.voronoi.data_ptr(), c.boxes.data_ptr(), None, c.n, c.hm,
                      c.wm, w, 128, 0.1, None, 0, hs, gs, rws.data_ptr(), rws.numel(), dev.stream_ptr())

    timings = {}
    for knob, values in KNOBS.items():
        best_v, best_t = get(knob), None
        for v in values:
            set(knob, v)
            t = _time(workload, repeats)
            timings[f"{knob}={v}"] = round(t, 4)
            if log:
                log(f"{knob}={v}: {t:.3f} ms")
            if best_t is None or t < best_t:
                best_v, best_t = v, t
        set(knob, best_v)
    out = {"config": current(), "ms": timings, "cells": int(cells.n)}
    if use_cache:
        cache[key] = out
        try:
            path.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return out
