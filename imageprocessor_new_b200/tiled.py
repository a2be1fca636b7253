"""Tiled centre detection with the page resident on the device (detect_centers(tile_h=...),
subpx/_gpu/centers.py:1778-1862): a global Otsu threshold of img[::ds, ::ds] x thr_scale, bands of
tile_h rows stepping tile_h - overlap, the keep-band rule, then a GPU dedupe (O(N) with a bin grid)
in place of the reference's O(N^2) Python loop.

With the global threshold, each band's pipeline (binarise, optional open / close, CCL, area filter,
refiners) is captured once as a CUDA graph over fixed buffers and replayed for every band of the
same height: the band is copied into the graph's input buffer, the counts stay on the device (the
refiners run over a fixed capacity of rows, those past the selected count giving NaN centres that
the keep rule drops), and the host reads the per-band component counts once at the end. The
capacity is twice the components of the band the graph was built on; a page with a band of more
components than that is redone by the eager path (and the graph rebuilt on the next call)."""

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


# Component capacity of a captured band: twice the components of the band it is built on (at least
# 1024, at most one per this many pixels); a page with a fuller band takes the eager path and the
# graph is rebuilt for the next call.
BAND_PX_PER_COMPONENT = 4


def band_capacity(band_h: int, width: int, components: int | None = None) -> int:
    most = max(1024, band_h * width // BAND_PX_PER_COMPONENT)
    return most if components is None else min(most, max(1024, 2 * int(components)))


class BandGraph:
    """The per-band pipeline of one band height, captured as a CUDA graph (see the module docstring)."""

    def __init__(self, band_h: int, width: int, dtype: torch.dtype, *, fixed_threshold: float, invert: bool,
                 area_min: int, area_max: int, pad: int, refine: str, connectivity: int, small_feature_max: float,
                 morph_open: int = 0, morph_close: int = 0, capacity: int | None = None,
                 sample: torch.Tensor | None = None):
        from .centers import _segmentation_source

        self.shape = (int(band_h), int(width))
        h, w = self.shape
        self.src = torch.zeros(self.shape, dtype=dtype, device="cuda")
        self.labels = dev.empty((h, w), torch.int32)
        self.count = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.kept = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.ccl_ws = dev.workspace(_lib.size("spx_ccl_workspace_bytes", h, w))
        self._seg = _segmentation_source
        self._seg_args = (float(fixed_threshold), bool(invert), int(morph_open), int(morph_close))
        if capacity is None and sample is not None:
            # Size the capacity on a real band: its component count, from the labelling alone.
            self.src.copy_(sample)
            src, thr, fixed, inv = self._seg(self.src, None, *self._seg_args)
            _lib.call("spx_ccl_label", src.data_ptr(), dev.dtype_code(src), h, w, dev.ptr(thr), float(fixed),
                      int(bool(inv)), int(connectivity), self.labels.data_ptr(), self.count.data_ptr(),
                      self.ccl_ws.data_ptr(), self.ccl_ws.numel(), dev.stream_ptr())
            capacity = band_capacity(h, w, dev.read_int(self.count))
        self.capacity = int(capacity) if capacity is not None else band_capacity(h, w)
        cap = self.capacity
        self.stats = dev.empty((cap + 1, 5), torch.int32)
        self.centroids = dev.empty((cap + 1, 2), torch.float64)
        self.rows = dev.empty((cap, 5), torch.int32)
        self.methods = dev.empty((cap,), torch.uint8)
        self.centers = dev.empty((cap, 2), torch.float64)
        self.sel_ws = dev.workspace(_lib.size("spx_select_workspace_bytes", cap))
        self._params = (int(area_min), int(area_max), int(pad), _lib.REFINE_CODES[refine], int(connectivity),
                        float(small_feature_max))
        self.graph = torch.cuda.CUDAGraph()
        self._launch()  # eager once: first launches and attribute settings happen outside the capture
        torch.cuda.synchronize()
        with torch.cuda.graph(self.graph):
            self._launch()

    def _launch(self):
        h, w = self.shape
        area_min, area_max, pad, refine, conn, sfm = self._params
        fixed, invert, mo, mc = self._seg_args
        src, thr, fixed, inv = self._seg(self.src, None, fixed, invert, mo, mc)
        stream = dev.stream_ptr()
        _lib.call("spx_ccl_label", src.data_ptr(), dev.dtype_code(src), h, w, dev.ptr(thr), float(fixed),
                  int(bool(inv)), conn, self.labels.data_ptr(), self.count.data_ptr(), self.ccl_ws.data_ptr(),
                  self.ccl_ws.numel(), stream)
        # Statistics for `capacity` labels: entries past the count stay empty (area 0), labels past
        # the capacity are not counted.
        _lib.call("spx_ccl_finish", self.labels.data_ptr(), h, w, conn, self.capacity, self.stats.data_ptr(),
                  self.centroids.data_ptr(), self.ccl_ws.data_ptr(), self.ccl_ws.numel(), stream)
        _lib.call("spx_select_components", self.stats.data_ptr(), self.capacity, area_min, area_max, refine, sfm,
                  self.rows.data_ptr(), self.methods.data_ptr(), self.kept.data_ptr(), self.sel_ws.data_ptr(),
                  self.sel_ws.numel(), stream)
        _lib.call("spx_refine_centers_counted", self.src.data_ptr(), dev.dtype_code(self.src), h, w,
                  self.labels.data_ptr(), self.rows.data_ptr(), self.methods.data_ptr(), self.kept.data_ptr(),
                  self.capacity, pad, self.centers.data_ptr(), stream)

    def run(self, band: torch.Tensor) -> torch.Tensor:
        """Replays the pipeline on `band` (same shape); returns the (capacity, 2) centres (NaN rows
        past the kept count) and leaves the band's component count in self.count."""
        self.src.copy_(band)
        self.graph.replay()
        return self.centers


_GRAPHS: dict = {}


def _keep_bands(bands, kept_rows):
    """The keep rule over (centres, y_offset, lo, hi) bands, appended on the device."""
    kept = dev.empty((max(kept_rows, 1), 2), torch.float64)
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    ws = dev.workspace(_lib.size("spx_keep_band_workspace_bytes", max((len(c) for c, *_ in bands), default=1)))
    for c, y_off, lo, hi in bands:
        if len(c):
            _lib.call("spx_keep_band", c.data_ptr(), len(c), float(y_off), float(lo), float(hi), kept.data_ptr(),
                      count.data_ptr(), max(kept_rows, 1), ws.data_ptr(), ws.numel(), dev.stream_ptr())
    return kept, count


def _bands_with_graphs(img_d, spans, pre, common):
    """Every band through a cached BandGraph of its height; None when a band overflows its capacity."""
    width = img_d.shape[1]
    graphs = {}
    keys = {}
    for y0, y1, _, _ in spans:
        key = (y1 - y0, width, img_d.dtype, float(pre), tuple(sorted(common.items())), torch.cuda.current_device(),
               BAND_PX_PER_COMPONENT)
        if key not in _GRAPHS:
            if len(_GRAPHS) >= 4:
                _GRAPHS.clear()
            _GRAPHS[key] = BandGraph(y1 - y0, width, img_d.dtype, fixed_threshold=pre, sample=img_d[y0:y1],
                                     **common)
        graphs[(y0, y1)] = _GRAPHS[key]
        keys[(y0, y1)] = key
    cap_total = sum(graphs[(y0, y1)].capacity for y0, y1, _, _ in spans)
    kept = dev.empty((max(cap_total, 1), 2), torch.float64)
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(len(spans), dtype=torch.int32, device="cuda")
    ws = dev.workspace(_lib.size("spx_keep_band_workspace_bytes", max(g.capacity for g in graphs.values())))
    for b, (y0, y1, lo, hi) in enumerate(spans):
        g = graphs[(y0, y1)]
        centers = g.run(img_d[y0:y1])
        counts[b:b + 1].copy_(g.count)
        _lib.call("spx_keep_band", centers.data_ptr(), g.capacity, float(y0), float(lo), float(hi), kept.data_ptr(),
                  count.data_ptr(), max(cap_total, 1), ws.data_ptr(), ws.numel(), dev.stream_ptr())
    over = [b for b, c in enumerate(counts.cpu().numpy()) if int(c) > graphs[spans[b][:2]].capacity]
    for b in over:  # rebuilt on the next call, sized on a band of this page
        _GRAPHS.pop(keys[spans[b][:2]], None)
    return None if over else (kept, count)


def detect_tiled(img, *, threshold, invert, area_min, area_max, pad, refine, connectivity, small_feature_max,
                 tile_h, overlap, threshold_mode, otsu_downsample, thr_scale, dedupe_eps, device, morph_open=0,
                 morph_close=0, use_graphs=True) -> CenterResult:
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
    spans = []
    y0 = 0
    while y0 < height:
        y1 = min(height, y0 + tile_h)
        half = overlap // 2
        lo = y0 if y0 == 0 else y0 + half
        hi = y1 if y1 == height else y1 - half
        spans.append((y0, y1, lo, hi))
        if y1 == height:
            break
        y0 += step
    common = dict(invert=invert, area_min=area_min, area_max=area_max, pad=pad, refine=refine,
                  connectivity=connectivity, small_feature_max=small_feature_max, morph_open=morph_open,
                  morph_close=morph_close)
    graphed = pre is not None and use_graphs
    out = _bands_with_graphs(img_d, spans, pre, common) if graphed else None
    if out is None:
        graphed = False
        bands = []
        for y0, y1, lo, hi in spans:
            band = img_d[y0:y1]
            thr = segment.binarize_threshold(band, threshold, invert) if pre is None else None
            c = _centers_on_device(band, threshold_dev=thr, fixed_threshold=pre if pre is not None else 0.0, **common)
            bands.append((c, y0, lo, hi))
        out = _keep_bands(bands, sum(len(c) for c, *_ in bands))
    kept, count = out
    n = dev.read_int(count)
    centers = _dedupe_device(kept[:n].contiguous(), n, float(dedupe_eps)).cpu().numpy() if n else np.zeros((0, 2))
    meta = {"tile_h": int(tile_h), "overlap": int(overlap), "threshold_mode": str(threshold_mode),
            "band_graphs": bool(graphed),
            "otsu_downsample": int(otsu_downsample), "thr_scale": float(thr_scale), "dedupe_eps": float(dedupe_eps),
            "refine": str(refine), "invert": bool(invert), "area_min": int(area_min), "area_max": int(area_max),
            "device": int(device), "small_feature_max": float(small_feature_max)}
    return CenterResult(centers_xy=centers, method=f"tiled_gpu(refine={refine})", backend="gpu", meta=meta)
