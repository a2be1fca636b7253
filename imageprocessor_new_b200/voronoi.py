"""Voronoi partition on the device (drop-in for subpx/_gpu/voronoi.py compute_voronoi_labels_gpu)."""

from __future__ import annotations

import numpy as np
import torch

from . import _device as dev
from . import _lib


def labels_device(seeds: torch.Tensor, shape) -> torch.Tensor:
    """(H, W) int32 device labels of the nearest seed; ``seeds`` is an (N, 2) float64 device tensor."""
    h, w = (int(v) for v in shape)
    n = int(seeds.shape[0]) if seeds is not None else 0
    out = dev.empty((h, w), torch.int32)
    ws = dev.workspace(_lib.size("spx_voronoi_workspace_bytes", n, h, w))
    _lib.call("spx_voronoi_labels", dev.ptr(seeds) if n else None, n, h, w, out.data_ptr(), ws.data_ptr(),
              ws.numel(), dev.stream_ptr())
    return out


def compute_voronoi_labels(seeds_xy: np.ndarray, image_shape, *, device: int = 0) -> np.ndarray:
    """Index of the nearest seed per pixel (exact ties to the lowest index), -1 without seeds
    (subpx/_gpu/voronoi.py:154-183)."""
    seeds = np.asarray(seeds_xy, dtype=np.float64)
    if seeds.size and (seeds.ndim != 2 or seeds.shape[1] != 2):
        raise ValueError(f"seeds_xy must be (N, 2), got {seeds.shape}")
    seeds = seeds.reshape(-1, 2)
    with dev.on_device(device):
        sd = dev.upload(seeds) if len(seeds) else None
        return labels_device(sd, image_shape).cpu().numpy()


compute_voronoi_labels_gpu = compute_voronoi_labels
