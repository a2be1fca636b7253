"""Oracle: the "projection" CD method -- CPU restatement, test infrastructure.

Follows subpx/_cpu/invariant_cd.py: _empty 308-317, _set_ellipses 320-336, _spline_operators 343-358
(scipy's not-a-knot CubicSpline of a profile padded with 32 zeros on both sides, sampled every 0.02
px with its slope) and _projection 365-421 (per cell the x and y profiles of the neighbour-removed
cell summed over its mask, the spline's highest point inside the profile's span, the steepest rise
before it and the steepest fall after it; width = their distance, centre = their midpoint; the
result is drawn as the axis-aligned ellipse of the two widths). Returns the oracle's measurement
dicts (centers, contours, status, metrics, edge_px).
"""

from __future__ import annotations

from functools import lru_cache

import numpy as np

ZERO_PAD = 32
NAMES = ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "perimeter_px", "background", "peak_signal")


@lru_cache(maxsize=16)
def spline_operators(size: int, step: float = 0.02):
    """(grid, value_op, slope_op): the spline of a profile p of `size` samples, padded with zeros, at
    the grid points is p @ value_op (size x len(grid)) and its slope p @ slope_op."""
    from scipy.interpolate import CubicSpline

    grid = np.arange(0.0, size - 1 + step / 2, step)
    n = size + 2 * ZERO_PAD
    unit = np.zeros((n, size))
    unit[ZERO_PAD + np.arange(size), np.arange(size)] = 1.0
    spline = CubicSpline(np.arange(n), unit, axis=0)
    return grid, spline(grid + ZERO_PAD).T.copy(), spline(grid + ZERO_PAD, 1).T.copy()


def ellipse_rows(out, rows, centers_local, cd_x, cd_y, origins, n_angles):
    """Axis-aligned ellipse of widths cd_x, cd_y about each centre: edge radii, contour, geometry."""
    out["centers"][rows] = centers_local + origins
    out["center_local"][rows] = centers_local
    a, b = cd_x / 2, cd_y / 2
    angles = np.arange(n_angles) * (2 * np.pi / n_angles)
    edge = a[:, None] * b[:, None] / np.sqrt((b[:, None] * np.cos(angles)) ** 2 + (a[:, None] * np.sin(angles)) ** 2)
    out["edge_px"][rows] = edge
    closed = np.concatenate([angles, angles[:1]])
    pts = centers_local[:, None, :] + edge[:, np.r_[np.arange(n_angles), 0], None] * \
        np.stack([np.cos(closed), np.sin(closed)], axis=1)[None]
    out["contours"][rows] = pts + origins[:, None, :]
    m = out["metrics"]
    m["cd_x_px"][rows], m["cd_y_px"][rows] = cd_x, cd_y
    m["area_px2"][rows] = np.pi * a * b
    m["cd_equivalent_px"][rows] = a + b
    h = ((a - b) / np.maximum(a + b, 1e-300)) ** 2
    m["perimeter_px"][rows] = np.pi * (a + b) * (1 + 3 * h / (10 + np.sqrt(4 - 3 * h)))


def projection(cleaned, masks, origins, n_angles=128, step=0.02):
    """The projection method on an (n, h, w) stack of neighbour-removed cells and their masks."""
    cleaned = np.asarray(cleaned, dtype=np.float64)
    masks = np.asarray(masks, dtype=bool)
    origins = np.asarray(origins, dtype=np.float64).reshape(-1, 2)
    n, h, w = masks.shape
    out = {"centers": np.full((n, 2), np.nan), "center_local": np.full((n, 2), np.nan),
           "contours": np.full((n, n_angles + 1, 2), np.nan), "edge_px": np.full((n, n_angles), np.nan),
           "status": np.full(n, "no_signal", dtype="U32"), "metrics": {k: np.full(n, np.nan) for k in NAMES}}
    widths, centers = np.full((n, 2), np.nan), np.full((n, 2), np.nan)
    good = np.zeros((n, 2), bool)
    cell = np.where(masks, cleaned, 0.0)
    out["metrics"]["peak_signal"][:] = np.where(masks, cleaned, -np.inf).reshape(n, -1).max(axis=1) if n else 0
    for axis, (size, sum_axis) in enumerate(((w, 1), (h, 2))):
        counts = masks.sum(axis=sum_axis)
        profile = cell.sum(axis=sum_axis)
        grid, value_op, slope_op = spline_operators(size, step)
        values, slope = profile @ value_op, profile @ slope_op
        index = np.arange(len(grid))
        for i in range(n):
            inside = np.flatnonzero(counts[i] > 0)
            if not len(inside):
                continue
            first, last = inside[0], inside[-1]
            span = (grid >= first) & (grid <= last)
            peak = np.argmax(np.where(span, values[i], -np.inf))
            left = np.argmax(np.where(span & (index <= peak), slope[i], -np.inf))
            right = np.argmin(np.where(span & (index >= peak), slope[i], np.inf))
            x_left, x_right = grid[left], grid[right]
            widths[i, axis] = x_right - x_left
            centers[i, axis] = (x_left + x_right) / 2
            good[i, axis] = not (x_left <= first or x_right >= last or not slope[i, left] > 0
                                 or not slope[i, right] < 0)
    signal = out["metrics"]["peak_signal"] > 0
    ok = signal & good.all(axis=1)
    out["status"][signal] = "edge_at_cell_border"
    out["status"][ok] = "ok"
    rows = np.flatnonzero(signal)
    ellipse_rows(out, rows, centers[rows], widths[rows, 0], widths[rows, 1], origins[rows], n_angles)
    for name in ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "perimeter_px"):
        out["metrics"][name][~ok] = np.nan
    return out
