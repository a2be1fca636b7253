"""Oracle: Voronoi labels and cell boxes (CPU restatement, test infrastructure).

subpx/_cpu/cells.py:8-33 assigns each pixel the nearest seed (cKDTree, two nearest), resolving exact
ties on recomputed squared distances by the lowest index: argmin over seeds of (d2, index) with
d2 = dx*dx + dy*dy rounded as NumPy rounds it. This restatement evaluates that rule directly on the
candidates a KD-tree returns within the nearest distance (plus one ulp).
"""

from __future__ import annotations

import numpy as np


def voronoi_labels(seeds_xy: np.ndarray, shape) -> np.ndarray:
    from scipy.spatial import cKDTree

    seeds = np.asarray(seeds_xy, dtype=np.float64).reshape(-1, 2)
    h, w = shape
    labels = np.full((h, w), -1, dtype=np.int32)
    if len(seeds) == 0:
        return labels
    if len(seeds) == 1:
        labels.fill(0)
        return labels
    tree = cKDTree(seeds)
    k = min(4, len(seeds))
    rows = max(1, 262144 // w)
    for y0 in range(0, h, rows):
        y1 = min(h, y0 + rows)
        yy, xx = np.mgrid[y0:y1, :w]
        pts = np.column_stack((xx.ravel(), yy.ravel())).astype(np.float64)
        dist, ids = tree.query(pts, k=k)
        # Exact squared distances of the returned candidates; ties by index.
        d2 = np.sum((seeds[ids] - pts[:, None, :]) ** 2, axis=2)
        order = np.argmin(np.where(d2 == d2.min(axis=1, keepdims=True), ids, np.iinfo(np.int64).max), axis=1)
        chosen = ids[np.arange(len(ids)), order]
        # A seed beyond the k returned can tie only when the k-th distance equals the nearest one.
        if k < len(seeds):
            for j in np.flatnonzero(dist[:, -1] <= np.nextafter(dist[:, 0], np.inf)):
                cand = np.asarray(tree.query_ball_point(pts[j], np.nextafter(dist[j, 0], np.inf)))
                dd = np.sum((seeds[cand] - pts[j]) ** 2, axis=1)
                chosen[j] = cand[dd == dd.min()].min()
        labels[y0:y1] = chosen.reshape(y1 - y0, w)
    return labels


def cell_boxes(rows, shape, pad: int):
    """Per-row cell box origin and size: x0 = max(0, int(x) - pad), x1 = min(W, int(x + w) + pad)
    (subpx/_cpu/cells.py:53-59; int() truncates toward zero)."""
    h, w = shape
    r = np.asarray(rows, dtype=np.float64).reshape(-1, 6)
    x0 = np.maximum(0, r[:, 0].astype(np.int32) - pad)
    y0 = np.maximum(0, r[:, 1].astype(np.int32) - pad)
    x1 = np.minimum(w, (r[:, 0] + r[:, 2]).astype(np.int32) + pad)
    y1 = np.minimum(h, (r[:, 1] + r[:, 3]).astype(np.int32) + pad)
    return np.column_stack((x0, y0)).astype(np.int32), np.column_stack((x1 - x0, y1 - y0)).astype(np.int32)


def cell_masks(labels: np.ndarray, origins: np.ndarray, sizes: np.ndarray) -> np.ndarray:
    """(N, Hm, Wm) bool stack: labels == j inside each cell's box (subpx/_gpu/cells.py:11-38)."""
    n = len(origins)
    if n == 0:
        return np.zeros((0, 0, 0), bool)
    hm, wm = int(sizes[:, 1].max()), int(sizes[:, 0].max())
    out = np.zeros((n, hm, wm), bool)
    for j in range(n):
        x0, y0 = origins[j]
        bw, bh = sizes[j]
        out[j, :bh, :bw] = labels[y0:y0 + bh, x0:x0 + bw] == j
    return out
