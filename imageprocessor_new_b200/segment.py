"""Segmentation on the device: Otsu threshold, binarisation, connected components with stats.

Device-level helpers take and return torch CUDA tensors; ``connected_components_stats`` is the
NumPy-facing drop-in for subpx/components.py:47-52 (``backend="gpu"``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _device as dev
from . import _lib
from .types import ComponentStatsResult


@dataclass
class Components:
    """Device labels (H, W) int32 (0 = background), stats (K+1, 5) int32, centroids (K+1, 2) f64."""

    labels: torch.Tensor
    stats: torch.Tensor
    centroids: torch.Tensor
    count: int  # K, components without the background


def otsu(img: torch.Tensor, step: int = 1) -> torch.Tensor:
    """Otsu threshold of img[::step, ::step] as a one-element device double (OpenCV THRESH_OTSU)."""
    h, w = img.shape
    code = dev.dtype_code(img)
    if code not in (0, 1):
        raise ValueError("Otsu thresholding needs a uint8 or uint16 image")
    out = dev.empty((1,), torch.float64)
    ws = dev.workspace(_lib.size("spx_otsu_workspace_bytes", code))
    _lib.call("spx_otsu", img.data_ptr(), code, h, w, int(step), out.data_ptr(), ws.data_ptr(), ws.numel(),
              dev.stream_ptr())
    return out


def triangle(img: torch.Tensor) -> torch.Tensor:
    """Triangle threshold of a uint8 image as a one-element device double (OpenCV THRESH_TRIANGLE)."""
    h, w = img.shape
    code = dev.dtype_code(img)
    if code != 0:
        raise ValueError("the triangle threshold needs a uint8 image (as OpenCV)")
    out = dev.empty((1,), torch.float64)
    ws = dev.workspace(_lib.size("spx_otsu_workspace_bytes", code))
    _lib.call("spx_triangle", img.data_ptr(), code, h, w, out.data_ptr(), ws.data_ptr(), ws.numel(),
              dev.stream_ptr())
    return out


def label(img: torch.Tensor, *, threshold: torch.Tensor | None = None, fixed_threshold: float = 0.0,
          invert: bool = False, connectivity: int = 8) -> Components:
    """Binarise (img > t, or img <= t with invert) and label 8/4-connected components, numbered as
    cv2.connectedComponentsWithStats numbers them, with their stats and centroids."""
    h, w = img.shape
    code = dev.dtype_code(img)
    labels = dev.empty((h, w), torch.int32)
    count = dev.empty((1,), torch.int32)
    ws = dev.workspace(_lib.size("spx_ccl_workspace_bytes", h, w))
    stream = dev.stream_ptr()
    _lib.call("spx_ccl_label", img.data_ptr(), code, h, w, dev.ptr(threshold), float(fixed_threshold),
              int(bool(invert)), int(connectivity), labels.data_ptr(), count.data_ptr(), ws.data_ptr(),
              ws.numel(), stream)
    k = dev.read_int(count)
    stats = dev.empty((k + 1, 5), torch.int32)
    centroids = dev.empty((k + 1, 2), torch.float64)
    _lib.call("spx_ccl_finish", labels.data_ptr(), h, w, int(connectivity), k, stats.data_ptr(),
              centroids.data_ptr(), ws.data_ptr(), ws.numel(), stream)
    return Components(labels, stats, centroids, k)


def binarize_threshold(img: torch.Tensor, threshold: str, invert: bool) -> torch.Tensor:
    """Automatic threshold value of `_segment_binary` (subpx/_cpu/centers.py:247-266)."""
    if threshold == "otsu":
        return otsu(img)
    if threshold == "triangle":
        return triangle(img)
    raise ValueError(f"Unsupported threshold method: {threshold!r}. Supported: ['otsu', 'triangle']")


def connected_components_stats(mask: np.ndarray, *, backend: str = "auto", connectivity: int = 8,
                               device: int = 0) -> ComponentStatsResult:
    """Labels, stats [x, y, w, h, area] and centroids of ``mask > 0`` (subpx/components.py:47-52)."""
    if backend not in ("auto", "gpu"):
        raise ValueError("imageprocessor_new_b200 runs on the GPU: backend must be 'gpu' or 'auto'")
    m = np.asarray(mask)
    if m.ndim != 2:
        raise ValueError("connected_components_stats expects a 2D mask.")
    if m.dtype == np.bool_:
        m = m.astype(np.uint8)
    if m.dtype not in _lib.DTYPES:
        m = (m > 0).astype(np.uint8)
    with dev.on_device(device):
        comp = label(dev.upload(m), fixed_threshold=0.0, connectivity=connectivity)
        return ComponentStatsResult(
            labels=comp.labels.cpu().numpy(), stats=comp.stats.cpu().numpy(),
            centroids=comp.centroids.cpu().numpy(), num_labels=comp.count + 1, backend="gpu",
            meta={"connectivity": int(connectivity), "implementation": "libsubpx_b200 union-find CCL"},
        )
