"""Tiled centre detection with the page resident on the device (detect_centers(tile_h=...),
subpx/_gpu/centers.py:1778-1862): a global Otsu threshold of img[::ds, ::ds] x thr_scale, bands of
tile_h rows stepping tile_h - overlap, the keep-band rule, then a GPU dedupe (O(N) with a bin grid)
in place of the reference's O(N^2) Python loop."""

from __future__ import annotations

import numpy as np
import torch

from . import _device as dev
from . import _lib
from . import segment
from .types import CenterResult


def dedupe_centers(centers_xy, *, eps: float = 1.5, device: int = 0) -> np.ndarray:
    """Merge near-duplicate centres (subpx/centers.py:335-378) on the GPU. Clusters come out in the
    order of their smallest member index."""
    pts = np.asarray(centers_xy, dtype=np.float64).reshape(-1, 2)
    if len(pts) == 0:
        return pts
    with dev.on_device(device):
        return _dedupe_device(dev.upload(pts), len(pts), float(eps)).cpu().numpy()


def _dedupe_device(pts_d: torch.Tensor, n: int, eps: float) -> torch.Tensor:
    lo = pts_d.min(dim=0).values.cpu().numpy()
    hi = pts_d.max(dim=0).values.cpu().numpy()
    args = (float(lo[0]), float(lo[1]), float(hi[0]), float(hi[1]), float(eps))
    ws = dev.workspace(_lib.size("spx_dedupe_workspace_bytes", n, *args))
    out = dev.empty((n, 2), torch.float64)
    count = dev.empty((1,), torch.int32)
    _lib.call("spx_dedupe_centers", pts_d.data_ptr(), n, *args, out.data_ptr(), count.data_ptr(), ws.data_ptr(),
              ws.numel(), dev.stream_ptr())
    return out[: dev.read_int(count)]


def detect_tiled(img, *, threshold, invert, area_min, area_max, pad, refine, connectivity, small_feature_max,
                 tile_h, overlap, threshold_mode, otsu_downsample, thr_scale, dedupe_eps, device, morph_open=0,
                 morph_close=0) -> CenterResult:
    from .centers import _centers_on_device, _device_image

    if overlap >= tile_h:
        raise ValueError("overlap must be < tile_h")
    if threshold_mode not in ("auto", "global", "per_tile"):
        raise ValueError("threshold_mode must be 'auto', 'global' or 'per_tile'")
    img_d = _device_image(img)
    height, width = img_d.shape
    pre = None
    if threshold_mode in ("global", "auto"):
        ds = max(1, int(otsu_downsample))
        pre = float(segment.otsu(img_d, step=ds).item()) * float(thr_scale)
    step = tile_h - overlap
    bands = []
    y0 = 0
    while y0 < height:
        y1 = min(height, y0 + tile_h)
        band = img_d[y0:y1]
        thr = segment.binarize_threshold(band, threshold, invert) if pre is None else None
        c = _centers_on_device(band, threshold_dev=thr, fixed_threshold=pre if pre is not None else 0.0,
                               invert=invert, area_min=area_min, area_max=area_max, pad=pad, refine=refine,
                               connectivity=connectivity, small_feature_max=small_feature_max,
                               morph_open=morph_open, morph_close=morph_close)
        half = overlap // 2
        lo = y0 if y0 == 0 else y0 + half
        hi = y1 if y1 == height else y1 - half
        bands.append((c, y0, lo, hi))
        if y1 == height:
            break
        y0 += step
    total = sum(len(c) for c, *_ in bands)
    kept = dev.empty((max(total, 1), 2), torch.float64)
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws = dev.workspace(_lib.size("spx_keep_band_workspace_bytes", max((len(c) for c, *_ in bands), default=1)))
    for c, y_off, lo, hi in bands:
        if len(c):
            _lib.call("spx_keep_band", c.data_ptr(), len(c), float(y_off), float(lo), float(hi), kept.data_ptr(),
                      count.data_ptr(), max(total, 1), ws.data_ptr(), ws.numel(), dev.stream_ptr())
    n = dev.read_int(count)
    centers = _dedupe_device(kept[:n].contiguous(), n, float(dedupe_eps)).cpu().numpy() if n else np.zeros((0, 2))
    meta = {"tile_h": int(tile_h), "overlap": int(overlap), "threshold_mode": str(threshold_mode),
            "otsu_downsample": int(otsu_downsample), "thr_scale": float(thr_scale), "dedupe_eps": float(dedupe_eps),
            "refine": str(refine), "invert": bool(invert), "area_min": int(area_min), "area_max": int(area_max),
            "device": int(device), "small_feature_max": float(small_feature_max)}
    return CenterResult(centers_xy=centers, method=f"tiled_gpu(refine={refine})", backend="gpu", meta=meta)
