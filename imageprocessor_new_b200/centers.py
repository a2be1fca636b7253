"""Centre detection on the device: threshold -> connected components -> per-blob refinement.

Drop-in for ``detect_centers(..., backend="gpu")`` of subpx/centers.py:130-220 and
``detect_centers_tiled`` (subpx/legacy.py:93-95). Semantics follow the reference CPU estimators
(subpx/_cpu/centers.py); see the module docstrings of csrc/refine.cu for the rules.
"""

from __future__ import annotations

import warnings

import numpy as np
import torch

from . import _device as dev
from . import _lib
from . import segment
from .types import CenterResult

_SUPPORTED_REFINE = ("none", "weighted", "logquad", "logquadratic", "edge_gradmoment", "edge_moment",
                     "edges_centered", "auto")
_VORONOI_METHODS = {"radial_symmetry", "isophote_curvature"}
# Refiners of ROI stacks, which detect_centers(background="model") can re-run on deblended cells
# (subpx/centers.py:34; the Voronoi refiners are outside this package).
_DEBLEND_METHODS = {"weighted", "logquad", "logquadratic", "none"}


def choose_refine_method_for_bbox(width: float, height: float, *, small_feature_max: float = 12.0) -> str:
    """logquad for features up to ``small_feature_max`` px, else edge_gradmoment (subpx/_cpu/centers.py:22-30)."""
    size = float(max(width, height))
    return "logquad" if size <= float(small_feature_max) else "edge_gradmoment"


def recommend_refine_method(width_px: float, height_px: float, *, small_feature_max: float = 12.0) -> str:
    return choose_refine_method_for_bbox(width_px, height_px, small_feature_max=small_feature_max)


def _check_backend(backend: str) -> None:
    if backend not in ("auto", "gpu"):
        raise ValueError("imageprocessor_new_b200 is the GPU backend: backend must be 'gpu' or 'auto'")


def _as_image(image):
    """NumPy array, or a CUDA tensor kept on the device."""
    if isinstance(image, torch.Tensor) and image.is_cuda:
        img = image
    else:
        img = image.detach().cpu().numpy() if isinstance(image, torch.Tensor) else np.asarray(image)
    if img.ndim != 2:
        raise ValueError("Expected 2D grayscale image.")
    return img


def _device_image(img) -> torch.Tensor:
    if isinstance(img, torch.Tensor):
        if img.dtype not in dev.TORCH_DTYPES.values():
            raise ValueError(f"unsupported image dtype {img.dtype}; use uint8, uint16, float32 or float64")
        return img.contiguous()
    if img.dtype not in _lib.DTYPES:
        raise ValueError(f"unsupported image dtype {img.dtype}; use uint8, uint16, float32 or float64")
    return dev.upload(img)


def _segmentation_source(img_d: torch.Tensor, threshold_dev, fixed_threshold: float, invert: bool, morph_open: int,
                         morph_close: int):
    """What segment.label binarises: the image itself, or (with morphology) the 0/255 image after
    cv2.morphologyEx OPEN / CLOSE with the 3x3 elliptic element (subpx/_cpu/centers.py:257-265)."""
    if not (morph_open or morph_close):
        return img_d, threshold_dev, fixed_threshold, invert
    h, w = img_d.shape
    bw = dev.empty((h, w), torch.uint8)
    tmp = dev.empty((h, w), torch.uint8)
    _lib.call("spx_binarize", img_d.data_ptr(), dev.dtype_code(img_d), h, w, dev.ptr(threshold_dev),
              float(fixed_threshold), int(bool(invert)), bw.data_ptr(), dev.stream_ptr())
    _lib.call("spx_morphology", bw.data_ptr(), h, w, int(morph_open), int(morph_close), tmp.data_ptr(),
              dev.stream_ptr())
    return bw, None, 0.0, False


def _centers_on_device(img_d: torch.Tensor, *, threshold_dev: torch.Tensor | None, fixed_threshold: float,
                       invert: bool, area_min: int, area_max: int, pad: int, refine: str,
                       connectivity: int, small_feature_max: float, morph_open: int = 0,
                       morph_close: int = 0) -> torch.Tensor:
    """Refined centres (n, 2) on the device, NaN rows for failed refinements, in label order."""
    src, thr, fixed, inv = _segmentation_source(img_d, threshold_dev, fixed_threshold, invert, morph_open,
                                                morph_close)
    comp = segment.label(src, threshold=thr, fixed_threshold=fixed, invert=inv, connectivity=connectivity)
    k = comp.count
    h, w = img_d.shape
    rows = dev.empty((max(k, 1), 5), torch.int32)
    methods = dev.empty((max(k, 1),), torch.uint8)
    kept = dev.empty((1,), torch.int32)
    ws = dev.workspace(_lib.size("spx_select_workspace_bytes", k))
    _lib.call("spx_select_components", comp.stats.data_ptr(), k, int(area_min), int(area_max),
              _lib.REFINE_CODES[refine], float(small_feature_max), rows.data_ptr(), methods.data_ptr(),
              kept.data_ptr(), ws.data_ptr(), ws.numel(), dev.stream_ptr())
    n = dev.read_int(kept)
    centers = dev.empty((max(n, 1), 2), torch.float64)
    _lib.call("spx_refine_centers", img_d.data_ptr(), dev.dtype_code(img_d), h, w, comp.labels.data_ptr(),
              rows.data_ptr(), methods.data_ptr(), n, int(pad), centers.data_ptr(), dev.stream_ptr())
    return centers[:n]


def _finite(centers: torch.Tensor) -> np.ndarray:
    """The finite rows of the device centres, through pinned host memory."""
    host = torch.empty(centers.shape, dtype=centers.dtype, pin_memory=True)
    host.copy_(centers, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    c = host.numpy().reshape(-1, 2)
    ok = np.isfinite(c[:, 0]) & np.isfinite(c[:, 1])
    return c if ok.all() else c[ok]


def detect_centers(
    image: np.ndarray,
    *,
    backend: str = "auto",
    threshold: str = "triangle",
    invert: bool = False,
    area_min: int = 1,
    area_max: int = 50,
    morph_open: int = 0,
    morph_close: int = 0,
    pad: int = 3,
    refine: str = "logquad",
    connectivity: int = 8,
    gpu_batch: int = 4096,
    device: int = 0,
    use_float64: bool = True,
    components_backend: str = "cpu",
    small_feature_max: float = 12.0,
    upsample_factor: int = 4,
    tile_h: int | None = None,
    overlap: int = 128,
    threshold_mode: str = "auto",
    otsu_downsample: int = 4,
    thr_scale: float = 0.8,
    dedupe_eps: float = 1.5,
    background: str | None = None,
    deblend_iterations: int = 30,
) -> CenterResult:
    """Detect and refine centres (subpx/centers.py:130-220), on the GPU.

    Centres are returned in component label order (the reference CPU order; the reference GPU
    path groups them by refine method). ``gpu_batch``, ``use_float64``, ``components_backend`` and
    ``upsample_factor`` are accepted for signature compatibility: every method runs in FP64 in one
    launch and components are always labelled on the GPU.
    """
    _check_backend(backend)
    if refine in _VORONOI_METHODS:
        raise NotImplementedError(f"refine='{refine}' is outside this package's hot path")
    if refine not in _SUPPORTED_REFINE:
        raise ValueError(f"Unsupported refine method: {refine}")
    if background not in (None, "model"):
        raise ValueError("background must be None or 'model'")
    if background == "model" and refine not in _DEBLEND_METHODS:
        raise NotImplementedError(
            f"background='model' is not supported for refine='{refine}': edge methods read the full image rather "
            "than per-cell ROIs. Use one of " + ", ".join(sorted(_DEBLEND_METHODS)) + ".")
    if connectivity not in (4, 8):
        raise ValueError("connectivity must be 4 or 8")
    if int(morph_open) < 0 or int(morph_close) < 0:
        raise ValueError("morph_open and morph_close must be >= 0")
    img = _as_image(image)
    if background == "model":
        result = detect_centers(img, backend=backend, threshold=threshold, invert=invert, area_min=area_min,
                                area_max=area_max, morph_open=morph_open, morph_close=morph_close, pad=pad,
                                refine=refine, connectivity=connectivity, gpu_batch=gpu_batch, device=device,
                                use_float64=use_float64, components_backend=components_backend,
                                small_feature_max=small_feature_max, upsample_factor=upsample_factor,
                                tile_h=tile_h, overlap=overlap, threshold_mode=threshold_mode,
                                otsu_downsample=otsu_downsample, thr_scale=thr_scale, dedupe_eps=dedupe_eps)
        with dev.on_device(device):
            return _refine_deblended(img, result, refine=refine, invert=invert, pad=int(pad),
                                     iterations=int(deblend_iterations), tile_h=tile_h, overlap=int(overlap))
    with dev.on_device(device):
        if tile_h is not None:
            return _detect_tiled(img, threshold=threshold, invert=invert, area_min=area_min, area_max=area_max,
                                 pad=pad, refine=refine, connectivity=connectivity,
                                 small_feature_max=small_feature_max, tile_h=int(tile_h), overlap=int(overlap),
                                 threshold_mode=threshold_mode, otsu_downsample=otsu_downsample,
                                 thr_scale=thr_scale, dedupe_eps=dedupe_eps, device=device,
                                 morph_open=int(morph_open), morph_close=int(morph_close))
        img_d = _device_image(img)
        thr = segment.binarize_threshold(img_d, threshold, invert)
        centers = _centers_on_device(img_d, threshold_dev=thr, fixed_threshold=0.0, invert=invert,
                                     area_min=area_min, area_max=area_max, pad=pad, refine=refine,
                                     connectivity=connectivity, small_feature_max=small_feature_max,
                                     morph_open=int(morph_open), morph_close=int(morph_close))
        arr = _finite(centers)
    meta = {
        "invert": bool(invert), "area_min": int(area_min), "area_max": int(area_max),
        "morph_open": int(morph_open), "morph_close": int(morph_close), "pad": int(pad),
        "connectivity": int(connectivity), "gpu_batch": int(gpu_batch), "device": int(device),
        "use_float64": bool(use_float64), "components_backend": str(components_backend),
        "small_feature_max": float(small_feature_max),
    }
    return CenterResult(centers_xy=arr, method=f"threshold={threshold}, refine={refine}", backend="gpu", meta=meta)


def _deblended_cells_centers(img_d: torch.Tensor, sign: float, seeds: np.ndarray, *, refine: str, pad: int,
                             iterations: int):
    """Centres of `seeds` re-refined on deblended cells (subpx/centers.py:224-268): square cells of
    2 ceil(0.6 pitch) + 1 around each seed cut by the Voronoi partition, a deblend of the image
    (background map and every hole's Gaussian), then the refiner on each cleaned cell restricted to
    its pixels above 0.2 x its peak. Returns (global centres with NaN rows, cell mask pixel counts,
    the deblend state)."""
    from .deblend import Deblender, auto_tile, build_cells

    h, w = (int(v) for v in img_d.shape)
    seeds_d = dev.upload(np.ascontiguousarray(seeds, dtype=np.float64))
    pitch = auto_tile(seeds_d, len(seeds), (h, w))[1]
    half = int(np.ceil(0.6 * pitch)) if np.isfinite(pitch) else 16
    rows = np.column_stack((seeds[:, 0] - half, seeds[:, 1] - half, np.full(len(seeds), 2 * half + 1.0),
                            np.full(len(seeds), 2 * half + 1.0), seeds[:, 0], seeds[:, 1])).reshape(-1, 6)
    cells = build_cells(rows, (h, w), pad)
    dbl = Deblender(img_d, sign, cells)
    state = dbl.run(iterations=iterations)
    n, hm, wm = cells.n, cells.hm, cells.wm
    if n == 0:
        return np.zeros((0, 2)), np.zeros(0, np.int64), state
    cleaned = dbl.cleaned(state)
    labels = dev.empty((n * hm, wm), torch.int32)
    refine_rows = dev.empty((n, 5), torch.int32)
    stream = dev.stream_ptr()
    _lib.call("spx_support_labels", cleaned.data_ptr(), cells.voronoi.data_ptr(), cells.boxes.data_ptr(),
              state.params_d.data_ptr(), n, hm, wm, w, labels.data_ptr(), refine_rows.data_ptr(), stream)
    methods = torch.full((n,), _lib.REFINE_CODES[refine], dtype=torch.uint8, device="cuda")
    local = dev.empty((n, 2), torch.float64)
    _lib.call("spx_refine_centers", cleaned.data_ptr(), _lib.DTYPES[np.dtype(np.float64)], n * hm, wm,
              labels.data_ptr(), refine_rows.data_ptr(), methods.data_ptr(), n, 0, local.data_ptr(), stream)
    centres = local.cpu().numpy()
    centres[:, 1] -= np.arange(n) * hm  # window row -> cell row
    centres += cells.origins
    return centres, cells.counts.cpu().numpy().astype(np.int64), state


def _refine_deblended(img, result: CenterResult, *, refine, invert, pad, iterations, tile_h, overlap) -> CenterResult:
    """detect_centers(background="model") (subpx/centers.py:271-314): the centres found without it
    re-refined on deblended cells, in row strips of tile_h (with +-overlap halos) when tiled."""
    sign = -1.0 if invert else 1.0
    seeds = np.asarray(result.centers_xy, dtype=np.float64).reshape(-1, 2)
    img_d = _device_image(img)
    height = img_d.shape[0]
    bands = [(0, height)] if not tile_h else [(y0, min(height, y0 + int(tile_h))) for y0 in range(0, height,
                                                                                                   int(tile_h))]
    centers, statuses, used, sources = [], [], 0, set()
    for y0, y1 in bands:
        lo, hi = (0, height) if not tile_h else (max(0, y0 - int(overlap)), min(height, y1 + int(overlap)))
        own = (seeds[:, 1] >= y0) & (seeds[:, 1] < y1)
        if not own.any():
            continue
        inside = (seeds[:, 1] >= lo) & (seeds[:, 1] < hi)
        found, _, state = _deblended_cells_centers(img_d[lo:hi].contiguous(), sign, seeds[inside] - [0, lo],
                                                   refine=refine, pad=pad, iterations=iterations)
        keep = own[inside]
        centers.append(found[keep] + [0, lo])
        statuses.append(state.status[keep])
        used = max(used, state.iterations)
        sources.add(state.background_info.get("source"))
    centers = np.concatenate(centers) if centers else np.zeros((0, 2))
    finite = np.isfinite(centers).all(axis=1)
    status = np.concatenate(statuses) if statuses else np.zeros(0, "U32")
    names, counts = np.unique(status, return_counts=True)
    meta = dict(result.meta)
    meta.update(background="model", deblend_iterations=int(iterations), deblend_iterations_used=int(used),
                deblend_status_counts=dict(zip(names.tolist(), counts.tolist())),
                background_source=sorted(s for s in sources if s), deblend_dropped_nonfinite=int((~finite).sum()))
    return CenterResult(centers_xy=centers[finite], method=result.method, backend=result.backend, meta=meta)


def _detect_tiled(img, *, threshold, invert, area_min, area_max, pad, refine, connectivity, small_feature_max,
                  tile_h, overlap, threshold_mode, otsu_downsample, thr_scale, dedupe_eps, device, morph_open=0,
                  morph_close=0) -> CenterResult:
    """Row bands of ``tile_h`` with an ``overlap`` halo, keep-band rule, dedupe
    (subpx/_gpu/centers.py:1778-1862), with the image resident on the device."""
    from . import tiled

    return tiled.detect_tiled(img, threshold=threshold, invert=invert, area_min=area_min, area_max=area_max,
                              pad=pad, refine=refine, connectivity=connectivity,
                              small_feature_max=small_feature_max, tile_h=tile_h, overlap=overlap,
                              threshold_mode=threshold_mode, otsu_downsample=otsu_downsample,
                              thr_scale=thr_scale, dedupe_eps=dedupe_eps, device=device, morph_open=morph_open,
                              morph_close=morph_close)


def detect_centers_tiled(image, *, tile_h=8192, **kwargs) -> CenterResult:
    """Deprecated alias of ``detect_centers(image, tile_h=...)`` (subpx/legacy.py:93-95)."""
    warnings.warn("detect_centers_tiled is deprecated; use detect_centers(image, tile_h=...)",
                  DeprecationWarning, stacklevel=2)
    kwargs.setdefault("backend", "gpu")
    return detect_centers(image, tile_h=tile_h, **kwargs)


def detect_centers_tiled_global_otsu(image, *, tile_h=8192, threshold_mode="global", **kwargs) -> CenterResult:
    warnings.warn("detect_centers_tiled_global_otsu is deprecated; use detect_centers(image, tile_h=..., "
                  "threshold_mode='global')", DeprecationWarning, stacklevel=2)
    kwargs.setdefault("backend", "gpu")
    return detect_centers(image, tile_h=tile_h, threshold_mode=threshold_mode, **kwargs)


def detect_centers_batch(frames, /, *args, progress: bool = False, **kwargs):
    """detect_centers over frames (subpx/batch.py:22-24)."""
    out = []
    for i, frame in enumerate(frames):
        out.append(detect_centers(frame, *args, **kwargs))
        if progress and (i + 1) % 50 == 0:
            print(f"processed {i + 1} frames")
    return out


def filter_centers(centers_xy, image_shape_hw, *, margin: float = 5.0) -> np.ndarray:
    """Centres at least ``margin`` px inside the image (subpx/centers.py:317-332)."""
    centers = np.asarray(centers_xy, dtype=np.float64)
    if centers.size == 0:
        return centers.reshape(0, 2)
    shape = tuple(image_shape_hw)
    h, w = int(shape[0]), int(shape[1])
    m = float(margin)
    x, y = centers[:, 0], centers[:, 1]
    keep = (x >= m) & (x < (w - m)) & (y >= m) & (y < (h - m))
    return centers[keep]
