"""measure_cds on the device: cells, deblending and CD measurements (drop-in for
``subpx.measure_cds(..., backend="gpu")``, subpx/cd.py:44-380 and _measure_cds 424-784).

Scope: ``background="model"`` with ``seeds="threshold"`` or ``seeds="peaks"``, ``smooth_sigma`` >= 0,
and the methods gaussian (deblended Gaussian FWHM), logquad, gradient and halfmax — the hot path.
Every per-pixel and per-cell step runs in libsubpx_b200; the host keeps the reference's
orchestration (validation, the seed revision bookkeeping, result assembly).
"""

from __future__ import annotations

import time

import numpy as np
import torch

from . import _device as dev
from . import _lib
from . import segment
from .deblend import FWHM_K, STATUS, Deblender, auto_tile, build_cells, sigma_major
from .types import CDMethodResult, CDResult, CDSummary

METHOD_LABELS = {
    "gaussian": "Deblended Gaussian FWHM",
    "logquad": "Gaussian FWHM",
    "gradient": "Maximum radial gradient",
    "halfmax": "Half-height contour",
    "projection": "x/y projection max-slope width",
    "half_area": "Area above half height",
    "half_area_min": "Area above half height (minimum level)",
    "half_area_min_avg": "Area above half height (minimum level, averaged peak)",
    "tail_area": "Area above a low threshold near the background",
    "tail_area_norm": "Area above a fraction of the peak (no background step)",
    "edge_area": "Area inside the steepest edge (no peak, no background step)",
    "foot_area": "Area inside the foot of the edge, a tail boundary (no peak, no background step)",
    "foot_area_ratio": "Area inside the foot of the edge, foot found once per image (no peak, no background step)",
}
# The half_area family: local level (median or minimum of the outermost pixels), averaged peak.
HALF_AREA = {"half_area": ("median", False), "half_area_min": ("min", False), "half_area_min_avg": ("min", True)}
# The tail family on windows of tail_window pitches: each one's threshold rule.
TAIL_AREA = {"tail_area": "median", "tail_area_norm": "zero", "edge_area": "edge", "foot_area": "foot",
             "foot_area_ratio": "given"}
AREA_METHODS = tuple(HALF_AREA) + tuple(TAIL_AREA)
SUPPORTED = tuple(METHOD_LABELS)
# Methods of the reference that are outside this package (invariant, local, outline families).
OTHER_METHODS = ("disk", "flux_ratio", "local_projection", "local_half_area", "local_half_area_min_avg",
                 "local_tail_area", "outline_fit", "outline_fit_fast")

GEOMETRY_METRICS = ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "perimeter_px")
FIT_METRICS = ("sigma_major_px", "sigma_minor_px", "fwhm_major_px", "fwhm_minor_px", "angle_deg", "log_fit_rmse")
# Device metric columns (include/subpx_b200.h): 0-4 geometry, 5 background, 6 peak_signal, 7.. method.
_COLS = GEOMETRY_METRICS + ("background", "peak_signal")


def _metric_names(method: str) -> tuple[str, ...]:
    if method == "logquad":
        return _COLS + FIT_METRICS
    if method == "gaussian":
        return _COLS + FIT_METRICS[:-1] + ("fit_rmse",)
    if method == "projection":
        return _COLS
    if method in AREA_METHODS:
        return _COLS + ("local_level", "threshold", "mean_signal") + (("steepest_level",) if method == "foot_area"
                                                                     else ())
    return _COLS + ("ray_coverage",)


_PROJECTION_STEP = 0.02
_ZERO_PAD = 32
_PROJECTION_OPS: dict = {}


def _projection_operators(size: int):
    """Grid length G and the (size, G) operators that give a profile's not-a-knot cubic spline and its
    slope at the points k * 0.02 (k < G) as profile @ operator: scipy's CubicSpline of the profile
    padded with 32 zeros on either side, as subpx/_cpu/invariant_cd.py:343-358 builds them (the spline
    is linear in the samples). Computed once per size on the host and kept on the device."""
    key = (int(size), torch.cuda.current_device())
    if key not in _PROJECTION_OPS:
        from scipy.interpolate import CubicSpline

        grid = np.arange(0.0, size - 1 + _PROJECTION_STEP / 2, _PROJECTION_STEP)
        n = size + 2 * _ZERO_PAD
        unit = np.zeros((n, size))
        unit[_ZERO_PAD + np.arange(size), np.arange(size)] = 1.0
        spline = CubicSpline(np.arange(n), unit, axis=0)
        value_op = np.ascontiguousarray(spline(grid + _ZERO_PAD).T)
        slope_op = np.ascontiguousarray(spline(grid + _ZERO_PAD, 1).T)
        _PROJECTION_OPS[key] = (len(grid), dev.upload(value_op), dev.upload(slope_op))
    return _PROJECTION_OPS[key]


_ZOOM_FACTOR = 4
_ZOOM_OPS: dict = {}


def _zoom_operator(size: int) -> torch.Tensor:
    """(size * 4, size) operator of the half_area family's enlargement along one axis: column i is
    scipy.ndimage.zoom (order 3, grid mode, zero outside) of the unit profile at i padded with 32
    zeros either side, cut back to the profile (subpx/_cpu/invariant_cd.py:424-444). On the device."""
    key = (int(size), torch.cuda.current_device())
    if key not in _ZOOM_OPS:
        from scipy.ndimage import zoom

        cols = []
        for i in range(size):
            e = np.zeros(size + 2 * _ZERO_PAD)
            e[_ZERO_PAD + i] = 1.0
            z = zoom(e, _ZOOM_FACTOR, order=3, mode="grid-constant", grid_mode=True)
            cols.append(z[_ZERO_PAD * _ZOOM_FACTOR:(_ZERO_PAD + size) * _ZOOM_FACTOR])
        _ZOOM_OPS[key] = dev.upload(np.ascontiguousarray(np.stack(cols, axis=1)))
    return _ZOOM_OPS[key]


def _validate(img, *, methods, background, seeds, threshold, area_min, area_max, pad, n_angles, radial_step,
              smooth_sigma, fit_fraction, deblend_iterations, deblend_tolerance, pixel_size, unit, metrics_only,
              summary_only, peak_min_distance, background_tile, background_level):
    """The reference's argument checks (subpx/cd.py:286-365), same messages."""
    if isinstance(img, torch.Tensor):
        if img.ndim != 2 or img.numel() == 0 or img.dtype not in dev.TORCH_DTYPES.values():
            raise ValueError("image must be a nonempty 2D real grayscale array")
        if img.dtype.is_floating_point and not bool(torch.isfinite(img).all()):
            raise ValueError("image must contain finite real intensities")
    else:
        if img.ndim != 2 or img.size == 0 or not np.issubdtype(img.dtype, np.number):
            raise ValueError("image must be a nonempty 2D real grayscale array")
        if np.iscomplexobj(img) or not np.isfinite(img).all():
            raise ValueError("image must contain finite real intensities")
    if background not in {"model", "border"}:
        raise ValueError("background must be 'model' or 'border'")
    if seeds not in {"threshold", "peaks"}:
        raise ValueError("seeds must be 'threshold' or 'peaks'")
    if seeds == "peaks" and background == "border":
        raise ValueError("seeds='peaks' requires background='model'")
    if methods is None:
        methods = ("gaussian", "logquad", "gradient", "halfmax") if background == "model" else (
            "logquad", "gradient", "halfmax")
    if isinstance(methods, str):
        methods = (methods,)
    methods = tuple(methods)
    known = SUPPORTED + OTHER_METHODS
    if not methods or len(set(methods)) != len(methods) or any(m not in known for m in methods):
        raise ValueError("methods must be unique choices from " + ", ".join(known))
    if "gaussian" in methods and background != "model":
        raise ValueError("method 'gaussian' requires background='model'")
    for name, value in (("metrics_only", metrics_only), ("summary_only", summary_only)):
        if not isinstance(value, (bool, np.bool_)):
            raise ValueError(f"{name} must be True or False")
    if not np.isfinite(deblend_tolerance) or deblend_tolerance <= 0:
        raise ValueError("deblend_tolerance must be positive")
    for name, value, lower in (("area_min", area_min, 1), ("area_max", area_max, area_min), ("pad", pad, 0),
                               ("n_angles", n_angles, 16), ("deblend_iterations", deblend_iterations, 1)):
        if not np.isfinite(value) or int(value) != value or value < lower:
            raise ValueError(f"{name} must be an integer >= {lower}")
    if not np.isfinite([radial_step, smooth_sigma, fit_fraction, pixel_size]).all():
        raise ValueError("measurement parameters must be finite")
    if not 0 < radial_step <= 1 or smooth_sigma < 0 or not 0 < fit_fraction < 1 or pixel_size <= 0:
        raise ValueError("require 0 < radial_step <= 1, smooth_sigma >= 0, 0 < fit_fraction < 1, pixel_size > 0")
    for name, value, lower in (("peak_min_distance", peak_min_distance, 1.0), ("background_tile", background_tile, 4)):
        if value is not None and (not np.isfinite(value) or value < lower):
            raise ValueError(f"{name} must be >= {lower}")
    if background_level is not None and not np.isfinite(background_level):
        raise ValueError("background_level must be finite")
    if not isinstance(unit, str) or not unit.strip():
        raise ValueError("unit must be a nonempty length-unit label")
    if unit == "px" and pixel_size != 1:
        raise ValueError("supply a physical unit when pixel_size differs from 1")
    return methods


def measure_cds(
    image: np.ndarray,
    *,
    methods: tuple[str, ...] | None = None,
    background: str = "model",
    seeds: str = "threshold",
    threshold: str = "otsu",
    invert: bool = False,
    area_min: int = 3,
    area_max: int = 50,
    pad: int = 3,
    n_angles: int = 128,
    radial_step: float = 0.1,
    smooth_sigma: float = 0.0,
    fit_fraction: float = 0.2,
    peak_min_distance: float | None = None,
    background_level: float | None = None,
    background_tile: int | None = None,
    deblend_iterations: int = 30,
    deblend_tolerance: float = 1e-3,
    pixel_size: float = 1.0,
    unit: str = "px",
    backend: str = "gpu",
    cell_backend: str | None = None,
    device: int = 0,
    metrics_only: bool = False,
    summary_only: bool = False,
    fit_precision: str = "fp64",
    half_area_level: float = 0.5,
    half_area_peak_pixels: float = 4.0,
    tail_area_level: float = 0.2,
    tail_window: float = 1.2,
    outlines: bool = True,
    **other,
) -> CDResult | CDSummary:
    """Voronoi cells and their CDs (subpx/cd.py:44-380) on the GPU.

    Cells, background map, Gaussian deblending and the gaussian / logquad / gradient / halfmax
    measurements follow the reference CPU path operation for operation (FP64). Parameters of the
    reference's other method families (``nominal_cd``, ``psf_fwhm``, ``tail_area_level``, ...) are
    accepted in ``other`` and must keep their defaults. ``projection``, the ``half_area`` family
    (``half_area_level``, ``half_area_peak_pixels``, ``outlines``) and the tail family (``tail_area``,
    ``tail_area_norm``, ``edge_area``, ``foot_area``, ``foot_area_ratio``; ``tail_area_level``,
    ``tail_window``) follow subpx/_cpu/invariant_cd.py; tail windows are limited to 64 px.

    ``fit_precision`` (no reference counterpart) sets the deblending LM's arithmetic: "fp64" is the
    reference's; "fp32" runs the per-pixel residuals, Jacobian and sums in FP32 (compensated J^T r
    and cost, FP64 totals) with the solve, acceptance and stop rule (relative cost drop 1e-7) in FP64.
    """
    on_device = isinstance(image, torch.Tensor) and image.is_cuda
    img = image if on_device else np.asarray(image.detach().cpu().numpy() if isinstance(image, torch.Tensor)
                                             else image)
    methods = _validate(img, methods=methods, background=background, seeds=seeds, threshold=threshold,
                        area_min=area_min, area_max=area_max, pad=pad, n_angles=n_angles, radial_step=radial_step,
                        smooth_sigma=smooth_sigma, fit_fraction=fit_fraction, deblend_iterations=deblend_iterations,
                        deblend_tolerance=deblend_tolerance, pixel_size=pixel_size, unit=unit,
                        metrics_only=metrics_only, summary_only=summary_only, peak_min_distance=peak_min_distance,
                        background_tile=background_tile, background_level=background_level)
    if not (np.isfinite(half_area_level) and 0 < half_area_level < 1):
        raise ValueError("half_area_level must be between 0 and 1")
    if not (np.isfinite(half_area_peak_pixels) and half_area_peak_pixels >= 1):
        raise ValueError("half_area_peak_pixels must be at least 1")
    if not (np.isfinite(tail_area_level) and 0 < tail_area_level < 1):
        raise ValueError("tail_area_level must be between 0 and 1")
    if not (np.isfinite(tail_window) and 0.5 <= tail_window <= 2):
        raise ValueError("tail_window must be between 0.5 and 2 pitches")
    if not isinstance(outlines, (bool, np.bool_)):
        raise ValueError("outlines must be True or False")
    from .deblend import fit_options

    fit_options(fit_precision)  # ValueError for an unknown arithmetic
    if backend not in {"cpu", "gpu", "auto"}:
        raise ValueError("backend must be 'cpu', 'gpu' or 'auto'")
    if cell_backend not in {None, "cpu", "gpu"}:
        raise ValueError("cell_backend must be 'cpu' or 'gpu'")
    if backend == "cpu" or cell_backend == "cpu":
        raise ValueError("imageprocessor_new_b200 is the GPU backend: use backend='gpu' (or 'auto')")
    if background != "model":
        raise ValueError("backend='gpu' requires background='model'; border mode runs on the CPU")
    unsupported = [m for m in methods if m not in SUPPORTED]
    if unsupported:
        raise NotImplementedError("methods outside the hot path: " + ", ".join(unsupported))
    metrics_only = bool(metrics_only) or bool(summary_only)
    with dev.on_device(device):
        return _measure_cds(img, methods=methods, threshold=threshold, invert=bool(invert), area_min=int(area_min),
                            area_max=int(area_max), pad=int(pad), n_angles=int(n_angles),
                            radial_step=float(radial_step), fit_fraction=float(fit_fraction),
                            background_level=background_level, background_tile=background_tile,
                            deblend_iterations=int(deblend_iterations), deblend_tolerance=float(deblend_tolerance),
                            pixel_size=float(pixel_size), unit=unit, device=int(device), metrics_only=metrics_only,
                            summary_only=bool(summary_only), fit_precision=fit_precision, seeds=seeds,
                            peak_min_distance=peak_min_distance, smooth_sigma=float(smooth_sigma),
                            half_area_level=float(half_area_level), half_area_peak_pixels=float(half_area_peak_pixels),
                            tail_area_level=float(tail_area_level), tail_window=float(tail_window),
                            outlines=bool(outlines))


def _segment(img_d: torch.Tensor, threshold: str, invert: bool):
    """Binary components of the reference's segmentation (subpx/cd.py:472-481): uint8 and uint16 +
    Otsu images are thresholded as they are, others are scaled to uint8 first."""
    rescaled = img_d.dtype != torch.uint8 and not (img_d.dtype == torch.uint16 and threshold == "otsu")
    seg = img_d
    if rescaled:
        gray = img_d.to(torch.float64)
        lo, hi = float(gray.min()), float(gray.max())
        span = hi - lo
        if span:
            seg = torch.round((gray - lo) * (255 / span)).to(torch.uint8)
        else:
            seg = torch.zeros(img_d.shape, dtype=torch.uint8, device="cuda")
    thr = segment.binarize_threshold(seg, threshold, invert)
    comp = segment.label(seg, threshold=thr, invert=invert, connectivity=8)
    return comp, rescaled


def _method_buffers(n: int, n_angles: int, method: str, contours: bool):
    """Every output of one method carved from ONE device buffer (256-byte aligned regions), so the
    result comes back in a single copy."""
    names = _metric_names(method)
    m = max(n, 1)
    shapes = {
        "centers": (m, 2),
        "contours": (m, n_angles + 1, 2) if contours else None,
        "metrics": (max(len(names), 13), m),  # column-major: one contiguous column per metric
        "center_local": (m, 2),
        "edge_px": (m, n_angles) if method in ("gradient", "halfmax") or (
            (method == "projection" or method in AREA_METHODS) and contours) else None,
        "eigenvalues": (m, 2) if method in ("logquad", "gaussian") else None,
        "axes": (m, 2, 2) if method in ("logquad", "gaussian") else None,
        "status": ((m + 7) // 8,),  # bytes, viewed as uint8
        "status_text": (m * 16,),   # 32 UCS-4 code points per cell, viewed on the host as "<U32"
    }
    offsets, total = {}, 0
    for key, shape in shapes.items():
        if shape is not None:
            offsets[key] = total
            total += -(-int(np.prod(shape)) // 32) * 32
    flat = dev.empty((total,), torch.float64)
    b = {"_flat": flat, "_layout": (shapes, offsets)}
    for key, shape in shapes.items():
        b[key] = None if shape is None else flat[offsets[key]:offsets[key] + int(np.prod(shape))].view(shape)
    b["status"] = b["status"].view(torch.uint8)[:m]
    struct = _lib.MethodOut(*(None if b[k] is None else b[k].data_ptr() for k in
                              ("centers", "contours", "status", "metrics", "center_local", "edge_px", "eigenvalues",
                               "axes")), b["metrics"].shape[0], m)
    return b, struct


_COPY_STREAMS: dict = {}


def _copy_stream() -> torch.cuda.Stream:
    dev_index = torch.cuda.current_device()
    if dev_index not in _COPY_STREAMS:
        _COPY_STREAMS[dev_index] = torch.cuda.Stream()
    return _COPY_STREAMS[dev_index]


def _start_download(b: dict, after: torch.cuda.Event):
    """Copies one method's buffer to pinned host memory on a side stream once `after` has fired;
    returns (host tensor, completion event)."""
    side = _copy_stream()
    side.wait_event(after)
    with torch.cuda.stream(side):
        h = torch.empty(b["_flat"].shape, dtype=torch.float64, pin_memory=True)
        h.copy_(b["_flat"], non_blocking=True)
        done = torch.cuda.Event()
        done.record(side)
    return h, done


def _to_result(method: str, n: int, b: dict, host: np.ndarray, metrics_only: bool, n_angles: int) -> CDMethodResult:
    names = _metric_names(method)
    shapes, offsets = b["_layout"]

    def part(key):
        shape = shapes[key]
        return host[offsets[key]:offsets[key] + int(np.prod(shape))].reshape(shape)[:n]

    shape = shapes["metrics"]
    m = host[offsets["metrics"]:offsets["metrics"] + int(np.prod(shape))].reshape(shape)
    codes = host[offsets["status"]:].view(np.uint8)[:n]
    # spx_status_text wrote the names on the device; the host only views them.
    status = host[offsets["status_text"]:offsets["status_text"] + shapes["status_text"][0]].view(
        np.dtype("<U32"))[:n]
    metrics = {name: m[k, :n] for k, name in enumerate(names)}
    if shapes["contours"] is not None:
        contours = part("contours")
    else:
        contours = np.empty((n, 0 if metrics_only else n_angles + 1, 2))
    geometry = {}
    if method == "logquad":
        geometry = {"center_local": part("center_local"), "eigenvalues": part("eigenvalues"), "axes": part("axes")}
    elif method in ("gradient", "halfmax"):
        geometry = {"center_local": part("center_local"), "edge_px": part("edge_px")}
    elif method == "projection" or method in AREA_METHODS:
        geometry = {"center_local": part("center_local"),
                    "edge_px": part("edge_px") if shapes["edge_px"] is not None else np.empty((n, 0))}
    elif not metrics_only:
        geometry = {"eigenvalues": part("eigenvalues"), "axes": part("axes")}
    return CDMethodResult(method=method, centers_xy=part("centers"), contours_xy=contours,
                          valid=codes == 0, status=status, metrics=metrics, geometry=geometry)


def _revise_seeds(dbl: Deblender, state, seeds_xy, pitch, oversized_d, *, drop_fraction=0.3, add_fraction=0.5):
    """Seeds to drop and holes to add after one deblending pass (subpx/_cpu/deblend.py:525-567)."""
    p = state.params
    # The median amplitude of the "ok" cells with A > 0 was taken on the device at the end of the
    # pass ("ok" implies finite params).
    reference = state.amplitude_median
    if not np.isfinite(reference):
        return np.zeros(len(p), bool), np.zeros((0, 2))
    h, w = dbl.shape
    resid = dev.empty((h, w), torch.float64)
    _lib.call("spx_residual", dbl.img.data_ptr(), dbl.dtype, dbl.sign, h, w, state.background.struct(),
              state.model.data_ptr(), resid.data_ptr(), dev.stream_ptr())
    sigma = max(0.5, 0.1 * pitch)
    radius_g = int(4.0 * sigma + 0.5)
    x = np.arange(-radius_g, radius_g + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    weights = dev.upload(phi / phi.sum())
    tmp = dev.empty((h, w), torch.float64)
    smooth = dev.empty((h, w), torch.float64)
    _lib.call("spx_gaussian_filter", resid.data_ptr(), h, w, weights.data_ptr(), radius_g, tmp.data_ptr(),
              smooth.data_ptr(), dev.stream_ptr())
    radius = max(1, int(np.floor(0.5 * pitch)))
    maxf = resid  # reuse
    _lib.call("spx_maximum_filter", smooth.data_ptr(), h, w, radius, tmp.data_ptr(), maxf.data_ptr(),
              dev.stream_ptr())
    # Host work while the filters run.
    finite = np.isfinite(p).all(axis=1)
    drop = ~finite | (p[:, 0] < drop_fraction * reference)
    count = dev.empty((1,), torch.int32)
    cap = 1 << 16
    peaks = dev.empty((cap, 2), torch.int32)
    _lib.call("spx_find_peaks", smooth.data_ptr(), maxf.data_ptr(), dev.ptr(oversized_d), h, w,
              float(add_fraction * reference), peaks.data_ptr(), cap, count.data_ptr(), dev.stream_ptr())
    k = dev.read_int(count)
    if k > cap:
        peaks = dev.empty((k, 2), torch.int32)
        _lib.call("spx_find_peaks", smooth.data_ptr(), maxf.data_ptr(), dev.ptr(oversized_d), h, w,
                  float(add_fraction * reference), peaks.data_ptr(), k, count.data_ptr(), dev.stream_ptr())
    yx = peaks[:k].cpu().numpy().astype(np.int64)
    order = np.lexsort((yx[:, 1], yx[:, 0]))  # np.nonzero order: row-major
    yx = yx[order]
    new = np.column_stack((yx[:, 1], yx[:, 0])).astype(float)
    n_kept = int(len(drop) - np.count_nonzero(drop))
    if len(new) and n_kept:
        # The kept seeds selected on the device from the cells' seeds (the same values as seeds_xy).
        kd = dbl.cells.seeds_d[dev.upload((~drop).view(np.uint8)).bool()]
        qd = dev.upload(np.ascontiguousarray(new))
        dist = dev.empty((len(new),), torch.float64)
        ws = dev.workspace(_lib.size("spx_voronoi_workspace_bytes", n_kept, h, w))
        _lib.call("spx_nearest_distances", kd.data_ptr(), n_kept, qd.data_ptr(), len(new), 0, h, w,
                  dist.data_ptr(), ws.data_ptr(), ws.numel(), dev.stream_ptr())
        new = new[dist.cpu().numpy() > 0.5 * pitch]
    return drop, new


def _peak_rows(img_d, sign, peak_min_distance):
    """Cell rows of peak seeds (subpx/cd.py:502-511): a (2 ceil(0.6 pitch) + 1)^2 box around each
    peak, no component, every hole reported by its fitted reach."""
    from . import peaks

    xy, pitch = peaks.detect_peaks(img_d, sign, min_distance=peak_min_distance)
    half = int(np.ceil(0.6 * pitch))
    rows = np.column_stack((xy[:, 0] - half, xy[:, 1] - half, np.full(len(xy), 2 * half + 1.0),
                            np.full(len(xy), 2 * half + 1.0), xy[:, 0], xy[:, 1])).reshape(-1, 6)
    return rows, pitch


def _measure_cds(img, *, methods, threshold, invert, area_min, area_max, pad, n_angles, radial_step, fit_fraction,
                 background_level, background_tile, deblend_iterations, deblend_tolerance, pixel_size, unit, device,
                 metrics_only, summary_only, fit_precision="fp64", seeds="threshold", peak_min_distance=None,
                 smooth_sigma=0.0, half_area_level=0.5, half_area_peak_pixels=4.0, tail_area_level=0.2,
                 tail_window=1.2, outlines=True):
    started = time.perf_counter()
    seconds = {}
    height, width = tuple(img.shape)
    sign = -1.0 if invert else 1.0
    if isinstance(img, torch.Tensor):
        img_d = img.contiguous()
    else:
        img_d = dev.upload(img if img.dtype in _lib.DTYPES else img.astype(np.float64))
    shape = tuple(img_d.shape)
    if seeds == "peaks":
        # Peak seeds (subpx/cd.py:502-511): no components, nothing excluded from the background, the
        # deblend's own tile, every hole reported by its fitted reach.
        rows, pitch = _peak_rows(img_d, sign, peak_min_distance)
        comp, rescaled, k, components_before_filter = None, False, 0, 0
        component_ids = np.full(len(rows), -1, np.int32)
        oversized_d = None

        def exclude_for(ids):
            return None

        cells = build_cells(rows, shape, pad)
        rows = cells.rows
        interior = np.ones(len(rows), bool)
        by_reach = np.ones(len(rows), bool)
        tile_px, tiled_seeds = None, None
    else:
        comp, rescaled = _segment(img_d, threshold, invert)
        k = comp.count
        components_before_filter = k
        # Area filter, cell rows, border flags and oversized labels on the device (subpx/cd.py:485-500).
        rows_d = dev.empty((max(k, 1), 6), torch.float64)
        ids_d = dev.empty((max(k, 1),), torch.int32)
        inside_d = dev.empty((max(k, 1),), torch.uint8)
        oversized_flags_d = dev.empty((k + 1,), torch.uint8)
        counts_d = dev.empty((2,), torch.int32)
        ws = dev.workspace(_lib.size("spx_select_workspace_bytes", k))
        _lib.call("spx_component_rows", comp.stats.data_ptr(), comp.centroids.data_ptr(), k, int(area_min), int(area_max),
                  width, height, rows_d.data_ptr(), ids_d.data_ptr(), inside_d.data_ptr(), oversized_flags_d.data_ptr(),
                  counts_d.data_ptr(), ws.data_ptr(), ws.numel(), dev.stream_ptr())
        n_keep, n_oversized = (int(v) for v in counts_d.cpu().numpy())
        rows_d = rows_d[:n_keep]
        # Host copies land while the Voronoi cells are built (build_cells syncs before reading them).
        rows = dev.start_download(rows_d)
        component_ids = dev.start_download(ids_d[:n_keep])
        interior_u8 = dev.start_download(inside_d[:n_keep])
        labels_d = comp.labels
        tmp8 = dev.empty((height, width), torch.uint8)
        oversized_d = None
        if n_oversized:
            oversized_d = dev.empty((height, width), torch.uint8)
            _lib.call("spx_label_mask", labels_d.data_ptr(), oversized_flags_d.data_ptr(), height, width, 0,
                      oversized_d.data_ptr(), tmp8.data_ptr(), dev.stream_ptr())

        def exclude_for(ids):
            flags = np.ones(k + 1, np.uint8)
            flags[0] = 0
            ids = ids[(ids >= 0) & (ids <= k)]
            flags[ids] = 0
            out = dev.empty((height, width), torch.uint8)
            flags_d = dev.upload(flags)  # held until the launch is queued (an upload freed earlier could be reused)
            _lib.call("spx_label_mask", labels_d.data_ptr(), flags_d.data_ptr(), height, width, 2,
                      out.data_ptr(), tmp8.data_ptr(), dev.stream_ptr())
            return out

        cells = build_cells(rows, shape, pad, rows_d=rows_d)
        rows = cells.rows
        interior = interior_u8.view(np.bool_)  # 0 / 1 bytes
        by_reach = np.zeros(len(rows), bool)
        tile_px, pitch = auto_tile(cells.seeds_d, cells.n, shape)
        tiled_seeds = cells
    seconds["segmentation"] = time.perf_counter() - started
    meta = {
        "background": "model", "seeds": seeds, "threshold": threshold, "invert": bool(invert),
        "area_min": int(area_min), "area_max": int(area_max), "pad": int(pad), "n_angles": int(n_angles),
        "radial_step": float(radial_step), "smooth_sigma": float(smooth_sigma), "fit_fraction": float(fit_fraction),
        "cell_backend": "gpu", "measurement_backend": "gpu", "device": int(device),
        "metrics_only": bool(metrics_only), "summary_only": bool(summary_only),
        "deblend_tolerance": float(deblend_tolerance), "fit_precision": fit_precision,
        "segmentation_rescaled": bool(rescaled),
        "components_before_filter": int(components_before_filter),
        "coordinates": "global [x, y] pixels; images indexed [y, x]", "seconds": seconds,
    }
    start = time.perf_counter()
    level = None if background_level is None else sign * float(background_level)

    def make_deblender(cells_, tile):
        return Deblender(img_d, sign, cells_, exclude_d=exclude_for(component_ids), tile=tile,
                         background_level=level, tolerance=deblend_tolerance, fit_precision=fit_precision)

    def tile_for(cells_):
        if background_tile is not None or cells_ is not tiled_seeds:
            return background_tile
        return tile_px

    passes = []
    added = dropped = 0
    state = dbl = None
    for revision in range(3):
        final = revision == 2 or not np.isfinite(pitch)
        dbl = make_deblender(cells, tile_for(cells))
        state = dbl.run(iterations=deblend_iterations if final else min(10, deblend_iterations))
        passes.append(int(state.iterations))
        if final:
            break
        drop, new = _revise_seeds(dbl, state, cells.seeds, pitch, oversized_d)
        if not drop.any() and not len(new):
            if state.converged or state.iterations >= deblend_iterations:
                break
            state = dbl.run(iterations=deblend_iterations - state.iterations, init=state.params)
            passes.append(int(state.iterations))
            break
        keep_s = ~drop
        half = int(np.ceil(0.6 * pitch))
        rows = np.concatenate((rows[keep_s], np.array([[px - half, py - half, 2 * half + 1, 2 * half + 1, px, py]
                                                       for px, py in new], dtype=np.float64).reshape(-1, 6)))
        component_ids = np.concatenate((component_ids[keep_s], np.full(len(new), -1, np.int32)))
        interior = np.concatenate((interior[keep_s], np.ones(len(new), bool)))
        by_reach = np.concatenate((by_reach[keep_s], np.ones(len(new), bool)))
        added, dropped = added + len(new), dropped + int(drop.sum())
        cells = build_cells(rows, shape, pad)
    if by_reach.any():
        params = state.params[by_reach]
        centers = params[:, 1:3] + cells.origins[by_reach]
        reach = np.where(np.isfinite(params).all(axis=1), 2 * FWHM_K * sigma_major(params), np.inf)
        interior[by_reach] = ((centers[:, 0] - reach > 0) & (centers[:, 0] + reach < width - 1)
                              & (centers[:, 1] - reach > 0) & (centers[:, 1] + reach < height - 1))
    report = np.flatnonzero(interior).astype(np.int32)
    nr = len(report)
    cleaned = dbl.cleaned(state, report)
    report_d = dev.upload(report) if nr else None
    seconds["deblend"], start = time.perf_counter() - start, time.perf_counter()
    found = {}
    stream = dev.stream_ptr()
    c = cells
    radial = [m for m in methods if m in ("gradient", "halfmax")]
    bufs, pending = {}, []  # pending: (method names, host copies and their completion events)
    main = torch.cuda.current_stream()

    def launched(names):
        # Each method's results go to pinned host memory on a side stream as soon as its kernel is
        # done, so the host converts one method while the GPU still runs the next.
        for name in names:
            b = bufs[name]
            _lib.call("spx_status_text", b["status"].data_ptr(), nr, b["status_text"].data_ptr(), stream)
        ev = torch.cuda.Event()
        ev.record(main)
        pending.append((names, [_start_download(bufs[name], ev) for name in names]))

    t_gauss = time.perf_counter()
    if "gaussian" in methods and nr:
        gb2 = _method_buffers(nr, n_angles, "gaussian", not metrics_only)
        _lib.call("spx_gaussian_method", state.params_d.data_ptr(), state.status_d.data_ptr(), cleaned.data_ptr(),
                  c.voronoi.data_ptr(), c.boxes.data_ptr(), report_d.data_ptr(), nr, c.hm, c.wm, width, n_angles,
                  gb2[1], stream)
        bufs["gaussian"] = gb2[0]
        launched(["gaussian"])
    t_gauss = time.perf_counter() - t_gauss
    if "logquad" in methods and nr:
        lb = _method_buffers(nr, n_angles, "logquad", not metrics_only)
        _lib.call("spx_logquad_cd", cleaned.data_ptr(), c.voronoi.data_ptr(), c.boxes.data_ptr(), report_d.data_ptr(),
                  c.seeds_d.data_ptr(), nr, c.hm, c.wm, width, n_angles, fit_fraction, lb[1], stream)
        bufs["logquad"] = lb[0]
        launched(["logquad"])
    if radial and nr:
        hb = _method_buffers(nr, n_angles, "halfmax", not metrics_only) if "halfmax" in radial else (None, None)
        gb = _method_buffers(nr, n_angles, "gradient", not metrics_only) if "gradient" in radial else (None, None)
        smooth_w, smooth_r = None, 0
        if smooth_sigma > 0:
            from .peaks import gaussian_weights

            weights, smooth_r = gaussian_weights(smooth_sigma)
            smooth_w = dev.upload(weights)
        ws = dev.workspace(_lib.size("spx_radial_workspace_bytes", c.hm, c.wm, int(smooth_w is not None)))
        _lib.call("spx_radial_cd", cleaned.data_ptr(), c.voronoi.data_ptr(), c.boxes.data_ptr(), report_d.data_ptr(),
                  nr, c.hm, c.wm, width, n_angles, radial_step, dev.ptr(smooth_w), smooth_r,
                  None if hb[1] is None else hb[1], None if gb[1] is None else gb[1], ws.data_ptr(), ws.numel(),
                  stream)
        if hb[0] is not None:
            bufs["halfmax"] = hb[0]
        if gb[0] is not None:
            bufs["gradient"] = gb[0]
        launched([m for m in ("halfmax", "gradient") if m in bufs])
    seconds["radial"] = time.perf_counter() - start - t_gauss
    t_proj = time.perf_counter()
    if "projection" in methods and nr:
        pb = _method_buffers(nr, n_angles, "projection", not metrics_only)
        gx, vx, sx = _projection_operators(c.wm)
        gy, vy, sy = _projection_operators(c.hm)
        _lib.call("spx_projection_cd", cleaned.data_ptr(), c.voronoi.data_ptr(), c.boxes.data_ptr(),
                  report_d.data_ptr(), nr, c.hm, c.wm, width, n_angles, _PROJECTION_STEP, vx.data_ptr(),
                  sx.data_ptr(), gx, vy.data_ptr(), sy.data_ptr(), gy, pb[1], stream)
        bufs["projection"] = pb[0]
        launched(["projection"])
    seconds["projection"] = time.perf_counter() - t_proj
    half = [m for m in methods if m in HALF_AREA]
    t_half = time.perf_counter()
    if half and nr:
        zy, zx = _zoom_operator(c.hm), _zoom_operator(c.wm)
        ws = dev.workspace(_lib.size("spx_half_area_workspace_bytes", c.hm, c.wm, _ZOOM_FACTOR))
        big_px = c.hm * c.wm * _ZOOM_FACTOR * _ZOOM_FACTOR
        n_top = min(max(1, int(round(half_area_peak_pixels * _ZOOM_FACTOR * _ZOOM_FACTOR))), big_px)
        for kind in ("median", "min"):
            names = [m for m in half if HALF_AREA[m][0] == kind]
            if not names:
                continue
            outs = {}
            for m in names:
                hb_ = _method_buffers(nr, n_angles, m, not metrics_only)
                bufs[m] = hb_[0]
                outs[HALF_AREA[m][1]] = hb_[1]
            _lib.call("spx_half_area_cd", cleaned.data_ptr(), c.voronoi.data_ptr(), c.boxes.data_ptr(),
                      report_d.data_ptr(), nr, c.hm, c.wm, width, n_angles, zy.data_ptr(), zx.data_ptr(), _ZOOM_FACTOR,
                      float(half_area_level), int(kind == "median"), n_top, int(bool(outlines) and not metrics_only),
                      outs.get(False), outs.get(True), ws.data_ptr(), ws.numel(), stream)
            launched(names)
    seconds["half_area"] = time.perf_counter() - t_half
    tails = [m for m in methods if m in TAIL_AREA]
    if tails and nr:
        t_tail = time.perf_counter()
        tail_bufs = _tail_areas(img_d, sign, state, c, report, report_d, pitch, tails, n_angles=n_angles,
                                level=tail_area_level, peak_pixels=half_area_peak_pixels, window=tail_window,
                                outlines=bool(outlines) and not metrics_only, metrics_only=metrics_only, meta=meta)
        bufs.update(tail_bufs)
        launched(tails)
        seconds["tail_area"] = time.perf_counter() - t_tail
    for names, copies in pending:
        t0 = time.perf_counter()
        for name, (host, done) in zip(names, copies):
            done.synchronize()
            found[name] = _to_result(name, nr, bufs[name], host.numpy(), metrics_only, n_angles)
        key = names[0] if names[0] in ("gaussian", "projection") else "half_area" if names[0] in HALF_AREA \
            else "tail_area" if names[0] in TAIL_AREA else "radial"
        seconds[key] = seconds.get(key, 0.0) + time.perf_counter() - t0
    seconds["gaussian"] = seconds.get("gaussian", 0.0) + t_gauss
    for name in methods:
        if not nr:
            found[name] = _empty_result(name, n_angles, metrics_only)
    found = {name: found[name] for name in methods}
    start = time.perf_counter()
    local_background = (state.background.at_points(c.seeds_d[dev.upload(report.astype(np.int64))], sign)
                        if nr else np.zeros(0))
    measurements = {}
    for name in methods:
        found[name].metrics["background"][:] = local_background
        measurements[name] = found[name]
    code_counts = np.bincount(state.status_codes[report], minlength=len(STATUS))
    present = sorted((str(STATUS[code]), int(cnt)) for code, cnt in enumerate(code_counts) if cnt)
    statuses, counts = np.array([name for name, _ in present]), np.array([cnt for _, cnt in present])
    info = state.background_info
    meta.update(
        background_definition=("Smooth map fitted jointly with one 2-D Gaussian per hole; measured cells have the map "
                               "and all other holes' models removed"),
        background_source=info.get("source"), background_tiles=info.get("tiles"),
        background_measured_tiles=info.get("measured_tiles"), background_tile_px=int(state.tile_px),
        background_level=background_level, deblend_iterations=int(deblend_iterations),
        deblend_iterations_used=sum(passes), deblend_passes=len(passes), deblend_pass_iterations=passes,
        deblend_converged=bool(state.converged),
        deblend_status_counts=dict(zip(statuses.tolist(), counts.tolist())), modelled_holes=int(len(rows)),
        seeds_added_from_residual=int(added), seeds_dropped_as_insignificant=int(dropped),
        pitch_px=float(pitch) if np.isfinite(pitch) else None,
        cell_stack_shape=[int(c.hm), int(c.wm)],
    )
    if summary_only:
        result = CDSummary(seeds_xy=c.seeds[report], measurements=measurements, pixel_size=float(pixel_size),
                           unit=unit, meta=meta)
        seconds["result"] = time.perf_counter() - start
        seconds["total"] = time.perf_counter() - started
        return result
    vor = c.voronoi.cpu().numpy()
    remap = np.full(len(rows) + 1, -1, dtype=np.int32)
    remap[report] = np.arange(nr, dtype=np.int32)
    cell_labels = remap[vor]
    params_global = state.params.copy()
    params_global[:, 1:3] += c.origins
    deblend_model = {"params": params_global, "report": report.astype(np.int64), "tile_px": int(state.tile_px)}
    if "tile_medians" in info:
        deblend_model["tile_medians"] = info["tile_medians"]
    if metrics_only:
        rois, masks = np.empty((nr, 0, 0)), np.empty((nr, 0, 0), bool)
    else:
        rois = cleaned.cpu().numpy()
        masks = _mask_stack(c, report)
    result = CDResult(
        image=img_d.cpu().numpy() if isinstance(img, torch.Tensor) else img.copy(),
        binary=np.zeros(shape, bool) if comp is None else comp.labels.cpu().numpy() > 0,
        component_labels=np.zeros(shape, np.int32) if comp is None else comp.labels.cpu().numpy(),
        component_ids=np.asarray(component_ids, dtype=np.int32)[report],
        boxes_xywh=rows[report, :4].astype(np.int32), seeds_xy=c.seeds[report], cell_labels=cell_labels,
        cell_areas_px2=np.bincount(cell_labels[cell_labels >= 0], minlength=nr), origins_xy=c.origins[report],
        rois=rois, masks=masks, measurements=measurements, pixel_size=float(pixel_size), unit=unit,
        background_map=sign * state.background.host_map(), deblend_model=deblend_model, meta=meta,
    )
    seconds["result"] = time.perf_counter() - start
    seconds["total"] = time.perf_counter() - started
    return result


def _mask_stack(c, report) -> np.ndarray:
    """(n, hm, wm) masks: label == j inside each cell's box (subpx/_gpu/cells.py:31-36)."""
    h, w = c.voronoi.shape
    rep = torch.as_tensor(report, dtype=torch.int64, device="cuda")
    boxes = c.boxes.to(torch.int64)[rep]
    r = torch.arange(c.hm, device="cuda")
    col = torch.arange(c.wm, device="cuda")
    inside = (r[None] < boxes[:, 3:4])[:, :, None] & (col[None] < boxes[:, 2:3])[:, None, :]
    ys = torch.clamp(boxes[:, 1:2] + r[None], 0, h - 1)[:, :, None]
    xs = torch.clamp(boxes[:, 0:1] + col[None], 0, w - 1)[:, None, :]
    return (inside & (c.voronoi.to(torch.int64)[ys, xs] == rep[:, None, None])).cpu().numpy()


_TAIL_CHUNK_BYTES = 512 * 2**20  # window arrays (float32 share + three byte masks) per chunk of holes


def _method_out_rows(b: dict, start: int) -> _lib.MethodOut:
    """A method's output struct shifted to row `start` (metrics stay column-major with the full stride)."""
    def at(key):
        t = b[key]
        if t is None:
            return None
        return (t[:, start:] if key == "metrics" else t[start:]).data_ptr()

    return _lib.MethodOut(at("centers"), at("contours"), at("status"), at("metrics"), at("center_local"),
                          at("edge_px"), None, None, b["metrics"].shape[0], b["metrics"].shape[1])


def _nanmedian_device(v: torch.Tensor) -> float:
    """numpy's nanmedian of a device vector: the middle value, or the mean of the two middle ones."""
    v = v[~torch.isnan(v)]
    n = int(v.numel())
    if n == 0:
        return float("nan")
    v = torch.sort(v).values
    if n % 2:
        return float(v[n // 2])
    return float((v[n // 2 - 1] + v[n // 2]) / 2)


def _tail_areas(img_d, sign, state, c, report, report_d, pitch, names, *, n_angles, level, peak_pixels, window,
                outlines, metrics_only, meta):
    """The tail family of the reported holes (subpx/_cpu/invariant_cd.py:1009-1068): windows of
    ceil(window x pitch) px half-width holding each hole's share of the light (spx_wide_cells), then
    spx_tail_area_cd on them, in chunks of holes; foot_area_ratio takes a second pass with the median
    foot ratio of the first. Returns the methods' device buffers."""
    nr = len(report)
    # measure_invariant's pitch: the deblend's, else (fewer than two holes) the stack's larger side.
    pitch_t = float(pitch) if np.isfinite(pitch) else float(max(c.hm, c.wm))
    radius = int(np.ceil(window * pitch_t))
    side = 2 * radius + 1
    if side > 64:
        raise NotImplementedError(f"tail windows of {side} px (tail_window x pitch): at most 64 px are supported")
    params = state.params
    good_amp = params[np.isfinite(params).all(axis=1), 0]
    floor = 1e-3 * float(np.median(good_amp)) if good_amp.size else 1e-12
    zy = _zoom_operator(side)
    zx_t = zy.t().contiguous()  # one operator per axis (square windows)
    big_px = side * side * _ZOOM_FACTOR * _ZOOM_FACTOR
    n_top = min(max(1, int(round(peak_pixels * _ZOOM_FACTOR * _ZOOM_FACTOR))), big_px)
    first = [m for m in names if m != "foot_area_ratio"]
    if "foot_area_ratio" in names and "foot_area" not in first:
        first.append("foot_area")
    bufs = {m: _method_buffers(nr, n_angles, m, not metrics_only) for m in first + [m for m in names if m not in first]}
    h, w = state.model.shape
    n_all = c.n
    cell_org = c.boxes[report_d.to(torch.int64), :2].contiguous()
    chunk = max(1, min(nr, _TAIL_CHUNK_BYTES // (7 * side * side)))
    ws_wide = dev.workspace(_lib.size("spx_wide_cells_workspace_bytes", n_all, chunk, h, w, pitch_t))
    ws_tail = dev.workspace(_lib.size("spx_tail_area_workspace_bytes", side, _ZOOM_FACTOR, n_angles))
    win_cells = dev.empty((chunk, side, side), torch.float32)
    inside = dev.empty((chunk, side, side), torch.uint8)
    level_px = dev.empty((chunk, side, side), torch.uint8)
    territory = dev.empty((chunk, side, side), torch.uint8)
    win_org = dev.empty((chunk, 2), torch.int32)
    bg = state.background.struct()
    stream = dev.stream_ptr()

    def run(kinds, cuts=None):
        for s0 in range(0, nr, chunk):
            m = min(chunk, nr - s0)
            _lib.call("spx_wide_cells", img_d.data_ptr(), dev.dtype_code(img_d), float(sign), h, w, bg,
                      state.model.data_ptr(), state.params_d.data_ptr(), c.boxes.data_ptr(), n_all, c.hm, c.wm,
                      report_d[s0:].data_ptr(), m, radius, pitch_t, floor, win_cells.data_ptr(), inside.data_ptr(),
                      level_px.data_ptr(), territory.data_ptr(), win_org.data_ptr(), None, ws_wide.data_ptr(),
                      ws_wide.numel(), stream)
            outs = [(_method_out_rows(bufs[k][0], s0) if k in kinds else None)
                    for k in ("tail_area", "tail_area_norm", "edge_area", "foot_area", "foot_area_ratio")]
            _lib.call("spx_tail_area_cd", win_cells.data_ptr(), inside.data_ptr(), level_px.data_ptr(),
                      territory.data_ptr(), win_org.data_ptr(), cell_org[s0:].data_ptr(), m, side, n_angles,
                      zy.data_ptr(), zx_t.data_ptr(), _ZOOM_FACTOR, float(level), n_top, int(outlines),
                      None if cuts is None else cuts[s0:].data_ptr(), *outs, ws_tail.data_ptr(), ws_tail.numel(),
                      stream)

    run(first)
    meta["tail_window_px"] = int(side)
    if "foot_area_ratio" in names:
        fb = bufs["foot_area"][0]
        cols = _metric_names("foot_area")
        threshold = fb["metrics"][cols.index("threshold"), :nr]
        steepest = fb["metrics"][cols.index("steepest_level"), :nr]
        valid = fb["status"][:nr] == 0
        ratio = _nanmedian_device((threshold / steepest)[valid])
        meta["foot_ratio"] = ratio
        cuts = (ratio * steepest).contiguous()
        run(["foot_area_ratio"], cuts)
    return {m: bufs[m][0] for m in names}


def _empty_result(method, n_angles, metrics_only) -> CDMethodResult:
    names = _metric_names(method)
    geometry = {}
    if method == "logquad":
        geometry = {"center_local": np.zeros((0, 2)), "eigenvalues": np.zeros((0, 2)), "axes": np.zeros((0, 2, 2))}
    elif method in ("gradient", "halfmax"):
        geometry = {"center_local": np.zeros((0, 2)), "edge_px": np.zeros((0, n_angles))}
    elif method == "projection" or method in AREA_METHODS:
        geometry = {"center_local": np.zeros((0, 2)), "edge_px": np.zeros((0, 0 if metrics_only else n_angles))}
    elif not metrics_only:
        geometry = {"eigenvalues": np.zeros((0, 2)), "axes": np.zeros((0, 2, 2))}
    return CDMethodResult(method=method, centers_xy=np.zeros((0, 2)),
                          contours_xy=np.zeros((0, 0 if metrics_only else n_angles + 1, 2)),
                          valid=np.zeros(0, bool), status=np.zeros(0, "U32"),
                          metrics={name: np.zeros(0) for name in names}, geometry=geometry)
