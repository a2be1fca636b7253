"""Uneven image stacks: the initial LM fits of every cell of every image in one persistent launch.

A stack is an (N, H, W) device array whose images may differ in pitch, hole size and cell count.
Each image is segmented and partitioned into Voronoi cells on its own, exactly as a single page is
(Otsu threshold, 8-connected components, area filter, padded boxes; subpx/cd.py:472-538), and the
cells are then concatenated into one work list over the stack seen as an (N * H, W) image: image
i's boxes move down by i * H rows and its Voronoi labels up by the number of cells before it, so
stack cell j is box j intersected with label j inside its own image. Seeds stay in their image's
rows (adding i * H to a fractional coordinate would round it); the kernels find a cell's image from
its box row (``spx_fit_options.rows_per_image``). One ``spx_deblend_initial_warm`` launch fits all
cells from one device work queue, plain or started by the learned warm start (whose patches
replicate each image's own edges, ``spx_extract_patches_stack``). Cell for cell the results are
those of the per-image fits, bit for bit (subpx/_cpu/deblend.py:152-171 and 174-254 per image).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _device as dev
from . import warmstart as ws
from .deblend import Cells


@dataclass
class StackCells:
    """Cells of a stack over its (N * H, W) view; ``starts[i]:starts[i + 1]`` are image i's cells.
    Boxes (and rows' box y) are in stack rows, seeds (rows' centroids) in their own image's rows."""

    cells: Cells
    starts: np.ndarray
    images: int
    height: int

    @property
    def n(self) -> int:
        return self.cells.n

    def image_of(self, i: int) -> slice:
        return slice(int(self.starts[i]), int(self.starts[i + 1]))


def stack_view(stack_d: torch.Tensor) -> torch.Tensor:
    """The (N, H, W) stack as one (N * H, W) image (no copy)."""
    if stack_d.dim() != 3 or not stack_d.is_cuda or not stack_d.is_contiguous():
        raise ValueError("a stack is a contiguous (N, H, W) CUDA tensor")
    n, h, w = stack_d.shape
    return stack_d.view(n * h, w)


def stack_cells(stack_d: torch.Tensor, *, area_min: int = 10, area_max: int = 2000, pad: int = 3) -> StackCells:
    """Per-image cells of the stack, concatenated into stack coordinates (see the module docstring)."""
    stack_view(stack_d)
    n_img, h, w = stack_d.shape
    vor = dev.empty((n_img * h, w), torch.int32)
    parts = []
    starts = [0]
    for i in range(n_img):
        c = ws.page_cells(stack_d[i], area_min=area_min, area_max=area_max, pad=pad)
        torch.add(c.voronoi, starts[-1], out=vor[i * h:(i + 1) * h])
        c.voronoi = None  # the stack's copy is the one kept
        parts.append(c)
        starts.append(starts[-1] + c.n)
    shift = [i * h for i in range(n_img)]
    # Box rows in stack rows; centroids (the seeds) in their own image's rows.
    rows = np.concatenate([p.rows + np.array([0, s, 0, 0, 0, 0], np.float64) for p, s in zip(parts, shift)])
    boxes = torch.cat([p.boxes + torch.tensor([0, s, 0, 0], dtype=torch.int32, device="cuda")
                       for p, s in zip(parts, shift)])
    seeds_d = torch.cat([p.seeds_d for p in parts])
    counts = torch.cat([p.counts for p in parts])
    caps = torch.cat([p.caps for p in parts])
    origins = np.concatenate([p.origins + np.array([0, s], p.origins.dtype) for p, s in zip(parts, shift)])
    sizes = np.concatenate([p.sizes for p in parts])
    hm = max((p.hm for p in parts), default=0)
    wm = max((p.wm for p in parts), default=0)
    max_px = max((p.max_px for p in parts), default=1)
    cells = Cells(rows, rows[:, 4:6], seeds_d.contiguous(), vor, boxes.contiguous(), counts, caps, origins, sizes,
                  hm, wm, max_px)
    return StackCells(cells, np.asarray(starts, np.int64), n_img, h)


def initial_fits(stack_d: torch.Tensor, sc: StackCells, *, net: ws.WarmStartNet | None = None, max_iter: int = 30):
    """Initial fits of all cells of the stack in one launch (with the patches and the MLP before it
    when ``net`` is given): params (ROI-local), status, iterations, backgrounds, fallback flags."""
    view = stack_view(stack_d)
    warm, tol = None, 1e-12
    if net is not None:
        warm = ws.predict_init(net, view, 1.0, sc.cells.seeds_d, sc.cells.boxes, sc.n, images=sc.images)
        tol = net.cost_tol
    return ws.initial_fits(view, sc.cells, max_iter=max_iter, warm=warm, cost_tol=tol, rows_per_image=sc.height)


def synth_stack(images: int, size: int, seed: int = 0) -> torch.Tensor:
    """(images, size, size) uint16 stack of synthetic pages rendered on the device, each with its own
    pitch U(16, 40), hole diameter 0.4-0.6 x pitch, 5 % missing and 2 % merged holes."""
    stack = dev.empty((images, size, size), torch.uint16)
    for i in range(images):
        page, _ = ws.synth_page(seed * 1_000_003 + i, size)
        stack[i].copy_(page)
    return stack
