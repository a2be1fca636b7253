"""Oracle: centre refinement and detection (CPU restatement, test infrastructure).

Follows subpx/_cpu/centers.py: _bg_from_border (31-42), refine_weighted_centroid_cpu (45-64),
refine_logquadratic_cpu (67-107), the edge gradient-moment estimator (111-223), refine_centers_cpu
(225-244), detect_centers_cpu (281-408); the tiled driver of subpx/_gpu/centers.py:1778-1862 (global
Otsu of img[::ds, ::ds] x thr_scale, fixed-threshold bands, keep-band rule) and dedupe_centers of
subpx/centers.py:335-378 (clusters of points within eps, the mean of each).
"""

from __future__ import annotations

import numpy as np

from . import segment


def border_median(roi: np.ndarray, border: int = 2) -> float:
    """Median of the top and bottom ``border`` rows and the left and right ``border`` columns (full
    height, so the corner pixels count twice), or of the whole ROI when it is too small."""
    g = np.asarray(roi, dtype=np.float64)
    h, w = g.shape
    if h <= 2 * border or w <= 2 * border:
        return float(np.median(g))
    frame = np.concatenate([g[:border].ravel(), g[-border:].ravel(), g[:, :border].ravel(),
                            g[:, -border:].ravel()])
    return float(np.median(frame))


def weighted_centroid(roi: np.ndarray, mask: np.ndarray):
    g = np.asarray(roi, dtype=np.float64)
    m = np.asarray(mask, dtype=bool)
    if not m.any():
        return np.nan, np.nan
    w = np.where(m, g - border_median(g), 0.0)
    w = np.maximum(w, 0.0)
    s = w.sum()
    ys, xs = np.indices(g.shape, dtype=np.float64)
    if s <= 0:
        yy, xx = np.nonzero(m)
        return float(xx.mean()), float(yy.mean())
    return float((xs * w).sum() / s), float((ys * w).sum() / s)


def logquad_center(roi: np.ndarray, mask: np.ndarray):
    """Stationary point of the least-squares quadratic fit to log(g - bg) over the mask pixels."""
    g = np.asarray(roi, dtype=np.float64)
    m = np.asarray(mask, dtype=bool)
    if m.sum() < 6:
        return np.nan, np.nan
    v = (g - border_median(g))[m]
    if v.size == 0 or v.max() <= 0:
        return np.nan, np.nan
    z = np.log(np.maximum(v, 1e-9))
    yy, xx = np.nonzero(m)
    x, y = xx.astype(np.float64), yy.astype(np.float64)
    design = np.column_stack([x * x, y * y, x * y, x, y, np.ones_like(x)])
    a, b, c, d, e, _ = np.linalg.lstsq(design, z, rcond=None)[0]
    hess = np.array([[2 * a, c], [c, 2 * b]])
    if np.linalg.cond(hess) > 1e8:
        return np.nan, np.nan
    try:
        cx, cy = np.linalg.solve(hess, [-d, -e])
    except np.linalg.LinAlgError:
        return np.nan, np.nan
    h, w = g.shape
    if not (0 <= cx < w and 0 <= cy < h):
        return np.nan, np.nan
    return float(cx), float(cy)


def _smooth5(p: np.ndarray) -> np.ndarray:
    """Binomial (1 4 6 4 1)/16 smoothing with edge replication, in NumPy's operation order."""
    pad = np.concatenate([[p[0], p[0]], p, [p[-1], p[-1]]])
    return (pad[:-4] + 4 * pad[1:-3] + 6 * pad[2:-2] + 4 * pad[3:-1] + pad[4:]) * (1.0 / 16.0)


def _edge_position(prof: np.ndarray, base: float, power: float = 8.0, loc_rad: int = 3):
    if prof.size < 3:
        return np.nan
    d = np.abs(np.diff(prof))
    if not np.isfinite(d).any():
        return np.nan
    ip = int(np.nanargmax(d))
    ip0 = min(max(ip, loc_rad), max(loc_rad, d.size - 1 - loc_rad))
    jj = np.clip(np.arange(ip0 - loc_rad, ip0 + loc_rad + 1), 0, d.size - 1)
    wgt = np.power(np.maximum(d[jj], 0.0), power)
    sw = float(wgt.sum())
    if sw <= 1e-12:
        return np.nan
    return float(np.sum(wgt * (base + (jj + 0.5))) / sw)


def edge_moment_center(roi: np.ndarray, mask: np.ndarray, *, band_rad=4, edge_rad=10, passes=2, iters=2):
    """Edge midpoints from four smoothed edge profiles, re-centred twice (gradient-moment edges)."""
    g = np.asarray(roi, dtype=np.float64)
    m = np.asarray(mask, dtype=bool)
    if g.ndim != 2 or g.shape != m.shape or not m.any():
        return np.nan, np.nan
    ys, xs = np.nonzero(m)
    w = float(xs.max() - xs.min() + 1)
    h = float(ys.max() - ys.min() + 1)
    xc, yc = float(xs.mean()), float(ys.mean())
    H, W = g.shape
    band = np.arange(-band_rad, band_rad + 1)
    span = np.arange(-edge_rad, edge_rad + 1)

    def prof_x(x0, y):
        rows = np.clip(int(np.rint(y)) + band, 0, H - 1)
        cols = np.clip(int(x0) + span, 0, W - 1)
        p = g[rows[:, None], cols[None, :]].mean(axis=0)
        for _ in range(passes):
            p = _smooth5(p)
        return p, float(int(x0) - edge_rad)

    def prof_y(y0, x):
        cols = np.clip(int(np.rint(x)) + band, 0, W - 1)
        rows = np.clip(int(y0) + span, 0, H - 1)
        p = g[rows[:, None], cols[None, :]].mean(axis=1)
        for _ in range(passes):
            p = _smooth5(p)
        return p, float(int(y0) - edge_rad)

    for _ in range(iters):
        xl = int(np.rint(xc - 0.5 * (w - 1.0)))
        xr = int(np.rint(xc + 0.5 * (w - 1.0)))
        yt = int(np.rint(yc - 0.5 * (h - 1.0)))
        yb = int(np.rint(yc + 0.5 * (h - 1.0)))
        edges = [_edge_position(*prof_x(xl, yc)), _edge_position(*prof_x(xr, yc)),
                 _edge_position(*prof_y(yt, xc)), _edge_position(*prof_y(yb, xc))]
        if not np.all(np.isfinite(edges)):
            return np.nan, np.nan
        xc, yc = 0.5 * (edges[0] + edges[1]), 0.5 * (edges[2] + edges[3])
    if not (np.isfinite(xc) and np.isfinite(yc)):
        return np.nan, np.nan
    return float(xc), float(yc)


def choose_method(w: float, h: float, small_feature_max: float = 12.0) -> str:
    return "logquad" if float(max(w, h)) <= float(small_feature_max) else "edge_gradmoment"


def refine(roi, mask, method: str, small_feature_max: float = 12.0):
    if method == "auto":
        ys, xs = np.nonzero(mask)
        if xs.size == 0:
            return np.nan, np.nan
        method = choose_method(xs.max() - xs.min() + 1, ys.max() - ys.min() + 1, small_feature_max)
    if method == "weighted":
        return weighted_centroid(roi, mask)
    if method in ("logquad", "logquadratic"):
        return logquad_center(roi, mask)
    if method in ("edge_gradmoment", "edge_moment", "edges_centered"):
        return edge_moment_center(roi, mask)
    if method == "none":
        ys, xs = np.nonzero(mask)
        return (np.nan, np.nan) if xs.size == 0 else (float(xs.mean()), float(ys.mean()))
    raise ValueError(method)


def centers_from_components(g, labels, stats, num, *, area_min, area_max, pad, refine_method,
                            small_feature_max=12.0):
    """Refined centres in label order (NaN rows dropped), as detect_centers_cpu's per-label loop."""
    H, W = g.shape
    out = []
    for lab in range(1, num):
        x, y, w, h, area = (int(v) for v in stats[lab])
        if area < area_min or area > area_max:
            continue
        x0, y0 = max(0, x - pad), max(0, y - pad)
        x1, y1 = min(W, x + w + pad), min(H, y + h + pad)
        roi = g[y0:y1, x0:x1]
        mask = labels[y0:y1, x0:x1] == lab
        method = choose_method(w, h, small_feature_max) if refine_method == "auto" else refine_method
        cx, cy = refine(roi, mask, method, small_feature_max)
        if np.isfinite(cx) and np.isfinite(cy):
            out.append([x0 + cx, y0 + cy])
    return np.asarray(out, dtype=np.float64).reshape(-1, 2)


def detect_centers(image, *, threshold="otsu", invert=False, area_min=1, area_max=50, pad=3,
                   refine_method="logquad", connectivity=8, small_feature_max=12.0, fixed_threshold=None,
                   morph_open=0, morph_close=0):
    g = np.asarray(image)
    if fixed_threshold is None:
        t = segment.otsu_threshold(g) if threshold == "otsu" else segment.triangle_threshold(g)
    else:
        t = fixed_threshold
    fg = segment.binarize(g, t, invert)
    if morph_open or morph_close:
        fg = segment.morphology(fg, morph_open, morph_close)
    num, labels, stats, _ = segment.label_components(fg, connectivity)
    return centers_from_components(g, labels, stats, num, area_min=area_min, area_max=area_max, pad=pad,
                                   refine_method=refine_method, small_feature_max=small_feature_max)


def dedupe(points: np.ndarray, eps: float = 1.5) -> np.ndarray:
    """Clusters of points linked by distances <= eps, each replaced by its mean (members summed in
    index order); clusters ordered by their smallest member index."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree

    pts = np.asarray(points, dtype=np.float64).reshape(-1, 2)
    n = len(pts)
    if n == 0:
        return pts
    pairs = cKDTree(pts).query_pairs(float(eps), output_type="ndarray")
    # query_pairs uses <= r on the Euclidean distance; keep the reference's test on squared distances.
    if len(pairs):
        d2 = np.sum((pts[pairs[:, 0]] - pts[pairs[:, 1]]) ** 2, axis=1)
        pairs = pairs[d2 <= float(eps) ** 2]
    graph = coo_matrix((np.ones(len(pairs)), (pairs[:, 0], pairs[:, 1])) if len(pairs) else ([], ([], [])),
                       shape=(n, n))
    _, comp = connected_components(graph, directed=False)
    first = np.full(comp.max() + 1, n)
    np.minimum.at(first, comp, np.arange(n))
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    sums = np.zeros((len(order), 2))
    counts = np.zeros(len(order))
    np.add.at(sums, rank[comp], pts)
    np.add.at(counts, rank[comp], 1)
    return sums / counts[:, None]


def detect_tiled(image, *, tile_h, overlap=128, threshold_mode="auto", otsu_downsample=4, thr_scale=0.8,
                 dedupe_eps=1.5, invert=False, area_min=1, area_max=50, pad=3, refine_method="logquad",
                 connectivity=8, small_feature_max=12.0, threshold="otsu"):
    """The reference GPU tiled driver's rules: global Otsu of img[::ds, ::ds] x thr_scale, bands of
    tile_h rows stepping tile_h - overlap, keep y in [y0 + overlap//2, y1 - overlap//2) except at the
    image edges, then dedupe."""
    img = np.asarray(image)
    H = img.shape[0]
    pre = None
    if threshold_mode in ("global", "auto"):
        ds = max(1, int(otsu_downsample))
        pre = segment.otsu_threshold(np.ascontiguousarray(img[::ds, ::ds])) * float(thr_scale)
    step = tile_h - overlap
    kept = []
    y0 = 0
    while y0 < H:
        y1 = min(H, y0 + tile_h)
        c = detect_centers(img[y0:y1], threshold=threshold, invert=invert, area_min=area_min, area_max=area_max,
                           pad=pad, refine_method=refine_method, connectivity=connectivity,
                           small_feature_max=small_feature_max, fixed_threshold=pre)
        if len(c):
            c = c.copy()
            c[:, 1] += y0
            half = overlap // 2
            lo = y0 if y0 == 0 else y0 + half
            hi = y1 if y1 == H else y1 - half
            c = c[(c[:, 1] >= lo) & (c[:, 1] < hi)]
            if len(c):
                kept.append(c)
        if y1 == H:
            break
        y0 += step
    if not kept:
        return np.zeros((0, 2))
    return dedupe(np.vstack(kept), dedupe_eps)


def dedupe_pairwise(points: np.ndarray, eps: float = 1.5) -> np.ndarray:
    """The reference's own O(N^2) dedupe (subpx/centers.py:335-380): for each point, squared
    distances to every later point, union-find (path halving, union by rank) of pairs within eps,
    cluster means ordered by root index. Same clusters and means as ``dedupe`` (whose order is by
    smallest member); kept to time the reference's cost on the CPU baseline of the tiled page."""
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 2)
    n = len(pts)
    if n == 0:
        return pts
    parent = np.arange(n, dtype=np.int64)
    rank = np.zeros(n, dtype=np.int8)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return int(a)

    eps2 = float(eps) ** 2
    for i in range(n):
        d2 = np.sum((pts[i + 1:] - pts[i]) ** 2, axis=1)
        for j in np.flatnonzero(d2 <= eps2) + i + 1:
            ra, rb = find(i), find(int(j))
            if ra == rb:
                continue
            if rank[ra] < rank[rb]:
                parent[ra] = rb
            elif rank[ra] > rank[rb]:
                parent[rb] = ra
            else:
                parent[rb] = ra
                rank[ra] += 1
    roots = np.array([find(i) for i in range(n)])
    _, inv = np.unique(roots, return_inverse=True)
    sums = np.zeros((inv.max() + 1, 2))
    counts = np.zeros(inv.max() + 1)
    np.add.at(sums, inv, pts)
    np.add.at(counts, inv, 1)
    return sums / counts[:, None]


def detect_centers_model(image, *, refine_method="logquad", invert=False, pad=3, deblend_iterations=30, **kw):
    """detect_centers(background="model") without bands (subpx/centers.py:178-297): the centres of
    `detect_centers`, then per centre a square cell of 2 ceil(0.6 pitch) + 1 (pitch from auto_tile;
    16 when undefined) cut by the Voronoi partition, a deblend (background map and every other
    hole's Gaussian removed), and the refiner again on each cleaned cell with support = the cell's
    mask where the cleaned value exceeds 0.2 x its peak (the fitted amplitude, else the cell's
    maximum). Returns (finite centres, deblend state, non-finite count)."""
    from . import deblend as odb
    from . import voronoi as ov

    g = np.asarray(image)
    seeds = detect_centers(g, refine_method=refine_method, invert=invert, pad=pad, **kw)
    signal = g.astype(np.float64) * (-1.0 if invert else 1.0)
    pitch = odb.auto_tile(seeds, signal.shape)[1]
    half = int(np.ceil(0.6 * pitch)) if np.isfinite(pitch) else 16
    rows = np.array([[x - half, y - half, 2 * half + 1, 2 * half + 1, x, y] for x, y in seeds],
                    dtype=np.float64).reshape(-1, 6)
    labels = ov.voronoi_labels(seeds, signal.shape)
    origins, sizes = ov.cell_boxes(rows, signal.shape, pad)
    masks = ov.cell_masks(labels, origins, sizes)
    state = odb.deblend(signal, seeds, masks, origins, iterations=deblend_iterations)
    cleaned = state.cleaned
    p0 = state.params[:, 0]
    peak = np.where(np.isfinite(p0) & (p0 > 0), p0, np.where(masks, cleaned, -np.inf).reshape(len(seeds), -1).max(axis=1))
    support = masks & (cleaned > 0.2 * peak[:, None, None])
    local = np.array([refine(c, m, refine_method) for c, m in zip(cleaned, support)], dtype=np.float64).reshape(-1, 2)
    centres = local + origins
    finite = np.isfinite(centres).all(axis=1)
    return centres[finite], state, int((~finite).sum())
