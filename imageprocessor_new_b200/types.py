"""Result types of the reference API (subpx/types.py:8-13, 121-152, 242-298), field for field."""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np


@dataclass
class CenterResult:
    centers_xy: np.ndarray
    method: str
    backend: str = "cpu"
    meta: dict[str, Any] = field(default_factory=dict)


@dataclass
class ComponentStatsResult:
    labels: np.ndarray
    stats: np.ndarray
    centroids: np.ndarray
    num_labels: int
    backend: str = "cpu"
    meta: dict[str, Any] = field(default_factory=dict)


@dataclass
class CDMethodResult:
    """One contour per cell; invalid measurements keep their cell index (NaN geometry, a status)."""

    method: str
    centers_xy: np.ndarray
    contours_xy: np.ndarray
    valid: np.ndarray
    status: np.ndarray
    metrics: dict[str, np.ndarray]
    geometry: dict[str, np.ndarray] = field(default_factory=dict)
    inputs: dict[str, np.ndarray] = field(default_factory=dict)


@dataclass
class CDSummary:
    """Per-hole measurements without image, label maps or cell stacks (``summary_only=True``)."""

    seeds_xy: np.ndarray
    measurements: dict[str, CDMethodResult]
    pixel_size: float = 1.0
    unit: str = "px"
    meta: dict[str, Any] = field(default_factory=dict)


@dataclass
class CDResult:
    """Cells, per-method CDs and calibration of one image (reference ``CDResult``)."""

    image: np.ndarray
    binary: np.ndarray
    component_labels: np.ndarray
    component_ids: np.ndarray
    boxes_xywh: np.ndarray
    seeds_xy: np.ndarray
    cell_labels: np.ndarray
    cell_areas_px2: np.ndarray
    origins_xy: np.ndarray
    rois: np.ndarray
    masks: np.ndarray
    measurements: dict[str, CDMethodResult]
    pixel_size: float = 1.0
    unit: str = "px"
    background_map: np.ndarray | None = None
    deblend_model: dict[str, Any] | None = None
    meta: dict[str, Any] = field(default_factory=dict)
    mean_intensity: np.ndarray = field(init=False)

    def __post_init__(self):
        """Mean original intensity over each full Voronoi cell, without fill."""
        assigned = self.cell_labels >= 0
        totals = np.bincount(
            self.cell_labels[assigned], weights=self.image[assigned].astype(np.float64),
            minlength=len(self.seeds_xy),
        )
        self.mean_intensity = np.divide(
            totals, self.cell_areas_px2,
            out=np.full(len(self.seeds_xy), np.nan), where=self.cell_areas_px2 > 0,
        )
