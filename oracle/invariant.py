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


# ---------------------------------------------------------------------------- the half_area family
# subpx/_cpu/invariant_cd.py: _zoom_operators 424-444, _nearest_pixels 447-456, _grow 459-467,
# _connected_to_top 470-490 (the 8-connected part of the above-threshold pixels that holds the top
# pixel), _top_mean 493-499, _half_areas 551-799 on the CPU (one size bucket, chunks of
# 4096 * 196 // (h * w) cells), _regions_by_arrays 802-875 for the level backgrounds.

HALF_AREA = {"half_area": ("median", False), "half_area_min": ("min", False), "half_area_min_avg": ("min", True)}
HALF_NAMES = NAMES + ("local_level", "threshold", "mean_signal")
FACTOR = 4


@lru_cache(maxsize=16)
def zoom_operator(size: int, factor: int = FACTOR) -> np.ndarray:
    """(size * factor, size): column i is scipy.ndimage.zoom (order 3, grid mode, zero outside) of
    the unit profile at i, padded with 32 zeros either side, cut back to the profile's extent."""
    from scipy.ndimage import zoom

    cols = []
    for i in range(size):
        e = np.zeros(size + 2 * ZERO_PAD)
        e[ZERO_PAD + i] = 1.0
        z = zoom(e, factor, order=3, mode="grid-constant", grid_mode=True)
        cols.append(z[ZERO_PAD * factor:(ZERO_PAD + size) * factor])
    return np.stack(cols, axis=1)


def _grow8(region):
    """Dilation of a batch of boolean images by one pixel in the 8 directions."""
    rows = region.copy()
    rows[:, 1:] |= region[:, :-1]
    rows[:, :-1] |= region[:, 1:]
    out = rows.copy()
    out[:, :, 1:] |= rows[:, :, :-1]
    out[:, :, :-1] |= rows[:, :, 1:]
    return out


def _component_of(above, top):
    """Per image, the 8-connected component of `above` holding its pixel `top` (flat index)."""
    from scipy.ndimage import label

    k, h, w = above.shape
    out = np.zeros_like(above)
    for i in range(k):
        y, x = divmod(int(top[i]), w)
        if above[i, y, x]:
            lab, _ = label(above[i], structure=np.ones((3, 3), bool))
            out[i] = lab == lab[y, x]
    return out


def _ring_level(mask, cell, kind):
    """Local level: median or minimum of each cell's outermost mask pixels (mask pixels with a
    4-neighbour outside the mask or on the stack's edge)."""
    k = len(mask)
    inner = mask.copy()
    inner[:, 1:] &= mask[:, :-1]
    inner[:, :-1] &= mask[:, 1:]
    inner[:, :, 1:] &= mask[:, :, :-1]
    inner[:, :, :-1] &= mask[:, :, 1:]
    inner[:, [0, -1]] = False
    inner[:, :, [0, -1]] = False
    ring = mask & ~inner
    if kind == "median":
        import warnings

        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)  # all-NaN rows: no ring
            return np.nanmedian(np.where(ring, cell, np.nan).reshape(k, -1), axis=1)
    return np.where(ring, cell, np.inf).reshape(k, -1).min(axis=1)


def _ring_or_level(mask, cell, kind, level_mask):
    """Local level b of each cell: `kind` 'median' / 'min' of its outermost mask pixels, or with
    `level_mask` the median over those pixels inside the mask; 'zero' for the kinds without one."""
    k = len(mask)
    if kind == "zero":
        return np.zeros(k)
    if level_mask is None:
        return _ring_level(mask, cell, kind)
    import warnings

    ring = level_mask & mask
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        return np.nanmedian(np.where(ring, cell, np.nan).reshape(k, -1), axis=1)


def _core(big_mask, d):
    """Pixels whose +-d difference stencil lies in the enlarged mask, none within d of the edge."""
    core = big_mask.copy()
    for axis in (1, 2):
        for shift in (d, -d):
            core &= np.roll(big_mask, shift, axis=axis)
    core[:, :d] = core[:, -d:] = False
    core[:, :, :d] = core[:, :, -d:] = False
    return core


def _edge_cut(big, big_mask, d):
    """edge_area's threshold (subpx/_cpu/invariant_cd.py:818-833): the enlarged cell's mean with each
    pixel weighted by its steepness (central differences +-d sub-pixels, one original pixel)."""
    pad = np.pad(big, ((0, 0), (d, d), (d, d)), mode="edge")
    steep = np.sqrt(((pad[:, 2 * d:, d:-d] - pad[:, :-2 * d, d:-d]) / (2 * d * (1.0 / d))) ** 2
                    + ((pad[:, d:-d, 2 * d:] - pad[:, d:-d, :-2 * d]) / (2 * d * (1.0 / d))) ** 2)
    wgt = np.where(_core(big_mask, d), steep, 0.0)
    total = wgt.sum(axis=(1, 2))
    return np.where(total > 0, (wgt * big).sum(axis=(1, 2)) / np.where(total > 0, total, 1.0), np.inf)


def _foot_cut(big, big_mask, d, zone):
    """foot_area's threshold and steepest level (subpx/_cpu/invariant_cd.py:834-857): below the
    steepness-weighted mean (the steepest level), the mean weighted by the signed curvature."""
    s = 1.0 / d
    pad = np.pad(big, ((0, 0), (d, d), (d, d)), mode="edge")
    up, down = pad[:, 2 * d:, d:-d], pad[:, :-2 * d, d:-d]
    right, left = pad[:, d:-d, 2 * d:], pad[:, d:-d, :-2 * d]
    steep = np.sqrt(((up - down) / (2 * d * s)) ** 2 + ((right - left) / (2 * d * s)) ** 2)
    curve = (up + down - 2 * big) / (d * s) ** 2 + (right + left - 2 * big) / (d * s) ** 2
    core = _core(big_mask, d)
    if zone is not None:
        core &= zone
    wgt = np.where(core, steep, 0.0)
    total = wgt.sum(axis=(1, 2))
    steepest = (wgt * big).sum(axis=(1, 2)) / np.where(total > 0, total, 1.0)
    outer = core & (big < steepest[:, None, None])
    bend = np.where(outer, curve, 0.0).sum(axis=(1, 2))
    cut = np.where((total > 0) & (bend > 0),
                   np.where(outer, curve * big, 0.0).sum(axis=(1, 2)) / np.where(bend > 0, bend, 1.0), np.inf)
    return cut, steepest


def areas(cells, masks, origins, n_angles, specs, *, level_masks=None, zone_masks=None, outlines=True):
    """The area methods of subpx/_cpu/invariant_cd.py:551-875 on an (n, h, w) stack of cells (CPU
    path, one size bucket): `specs` are dicts of name, level, background ('median', 'min', 'zero',
    'edge', 'foot' or 'given'), peak_pixels (None: the highest enlarged pixel) and cuts (per-cell
    thresholds for 'given'). `level_masks`: per cell, the pixels the median local level is taken over
    (instead of the outermost pixels); `zone_masks`: foot's territory. Returns per name the oracle's
    measurement dict (metrics: the half_area names, plus steepest_level for 'foot')."""
    cells = np.asarray(cells, dtype=np.float64)
    masks = np.asarray(masks, dtype=bool)
    origins = np.asarray(origins, dtype=np.float64).reshape(-1, 2)
    n, h, w = masks.shape
    sy = sx = 1.0 / FACTOR
    shift = (FACTOR - 1) / (2 * FACTOR)
    zy, zx = zoom_operator(h), zoom_operator(w)
    H, W = zy.shape[0], zx.shape[0]
    iy, ix = np.arange(h).repeat(FACTOR), np.arange(w).repeat(FACTOR)
    gy, gx = np.arange(H, dtype=float), np.arange(W, dtype=float)
    angles = np.arange(n_angles) * (2 * np.pi / n_angles)
    radii = np.arange(0.0, float(np.hypot(h, w)), 0.125)
    cos_a, sin_a = np.cos(angles), np.sin(angles)
    out = {}
    for spec in specs:
        names = HALF_NAMES + (("steepest_level",) if spec["background"] == "foot" else ())
        out[spec["name"]] = {"centers": np.full((n, 2), np.nan), "center_local": np.full((n, 2), np.nan),
                             "contours": np.full((n, n_angles + 1, 2), np.nan),
                             "edge_px": np.full((n, n_angles), np.nan),
                             "status": np.full(n, "no_signal", dtype="U32"),
                             "metrics": {k: np.full(n, np.nan) for k in names}}
    chunk = max(1, 4096 * 196 // (h * w))
    for start in range(0, n, chunk):
        rows = np.arange(start, min(n, start + chunk))
        k = len(rows)
        mask = masks[rows]
        cell = np.where(mask, cells[rows], 0.0)
        big_mask = mask[:, iy][:, :, ix]
        lm = None if level_masks is None else np.asarray(level_masks, bool)[rows]
        levels, bigs, peaks = {}, {}, {}
        for spec in specs:
            name, level, background = spec["name"], spec["level"], spec["background"]
            kind = background if background in ("median", "min") else "zero"
            if kind not in levels:
                b = _ring_or_level(mask, cell, kind, lm)
                levels[kind] = b
                centered = np.where(mask, cell - b[:, None, None], 0.0)
                bigs[kind] = zy[None] @ centered @ zx.T[None]
            b, big = levels[kind], bigs[kind]
            flat = np.where(big_mask, big, -np.inf).reshape(k, -1)
            top = np.argmax(flat, axis=1)
            peak = flat[np.arange(k), top]
            if spec["peak_pixels"] is not None:
                n_top = min(max(1, int(round(spec["peak_pixels"] * FACTOR * FACTOR))), H * W)
                if (kind, n_top) not in peaks:
                    p = np.partition(flat, -n_top, axis=1)[:, -n_top:].mean(axis=1)
                    peaks[kind, n_top] = np.where(np.isfinite(p), p, -1.0)
                peak = peaks[kind, n_top]
            steepest = None
            if background == "edge":
                cut = _edge_cut(big, big_mask, FACTOR)
            elif background == "foot":
                zone = None if zone_masks is None else np.asarray(zone_masks, bool)[rows][:, iy][:, :, ix]
                cut, steepest = _foot_cut(big, big_mask, FACTOR, zone)
            elif background == "given":
                cut = np.asarray(spec["cuts"], dtype=float)[rows]
            else:
                cut = level * peak
            above = big_mask & (big > cut[:, None, None])
            region = _component_of(above, top)
            count = region.sum(axis=(1, 2))
            touches = ((_grow8(region) & ~big_mask).any(axis=(1, 2)) | region[:, [0, -1]].any(axis=(1, 2))
                       | region[:, :, [0, -1]].any(axis=(1, 2)))
            weight = np.maximum(count, 1)
            mean_signal = np.where(region, big, 0.0).sum(axis=(1, 2)) / weight
            cy = (region.sum(axis=2) * gy).sum(axis=1) / weight
            cx = (region.sum(axis=1) * gx).sum(axis=1) / weight
            var_x = (region.sum(axis=1) * (gx[None] - cx[:, None]) ** 2).sum(axis=1) / weight * sx * sx
            var_y = (region.sum(axis=2) * (gy[None] - cy[:, None]) ** 2).sum(axis=1) / weight * sy * sy
            cd_eq = 2 * np.sqrt(count * (sx * sy) / np.pi)
            ratio = np.sqrt(np.sqrt(np.maximum(var_x, 1e-12) / np.maximum(var_y, 1e-12)))
            o = out[name]
            signal = (peak > 0) & np.isfinite(cut) & (cut < peak)
            m = o["metrics"]
            m["local_level"][rows] = b
            m["peak_signal"][rows] = np.where(signal, peak, np.nan)
            m["threshold"][rows] = np.where(signal, b + cut, np.nan)
            m["mean_signal"][rows] = np.where(signal, mean_signal, np.nan)
            if steepest is not None:
                m["steepest_level"][rows] = np.where(signal, steepest, np.nan)
            m["area_px2"][rows] = np.where(signal, count * (sx * sy), np.nan)
            m["cd_x_px"][rows] = np.where(signal, cd_eq * ratio, np.nan)
            m["cd_y_px"][rows] = np.where(signal, cd_eq / ratio, np.nan)
            o["status"][rows] = np.where(~signal, "no_signal", np.where(touches, "region_at_cell_border", "ok"))
            o["center_local"][rows] = np.column_stack((cx * sx - shift, cy * sy - shift))
            if outlines:
                # The region's last pixel along each ray from its centroid, in 1/8 px steps.
                far = ((gx[None, None] - cx[:, None, None]) * sx) ** 2 + ((gy[None, :, None] - cy[:, None, None]) * sy) ** 2
                reach = float(np.sqrt(np.where(region, far, 0.0).max())) if k else 0.0
                steps = radii[:min(len(radii), int(reach / 0.125) + 3)]
                px = np.rint(cx[:, None, None] + cos_a[None, :, None] * steps[None, None] / sx).astype(np.int64)
                py = np.rint(cy[:, None, None] + sin_a[None, :, None] * steps[None, None] / sy).astype(np.int64)
                inside = (px >= 0) & (px < W) & (py >= 0) & (py < H)
                index = (np.clip(py, 0, H - 1) * W + np.clip(px, 0, W - 1)).reshape(k, -1)
                hit = np.take_along_axis(region.reshape(k, -1), index, axis=1).reshape(px.shape) & inside
                first_out = np.where(hit.all(axis=2), len(steps), np.argmin(hit, axis=2))
                o["edge_px"][rows] = steps[np.maximum(first_out - 1, 0)] + 0.0625
    for spec in specs:
        o = out[spec["name"]]
        m = o["metrics"]
        m["cd_equivalent_px"][:] = 2 * np.sqrt(m["area_px2"] / np.pi)
        rows = np.flatnonzero(o["status"] != "no_signal")
        o["center_local"][o["status"] == "no_signal"] = np.nan
        o["centers"][rows] = o["center_local"][rows] + origins[rows]
        if outlines:
            o["edge_px"][o["status"] == "no_signal"] = np.nan
            c = o["center_local"][rows]
            dirs = np.column_stack((cos_a, sin_a))
            pts = c[:, None, :] + o["edge_px"][rows][:, :, None] * dirs[None]
            o["contours"][rows] = np.concatenate((pts, pts[:, :1]), axis=1) + origins[rows][:, None, :]
            m["perimeter_px"][rows] = np.linalg.norm(np.diff(o["contours"][rows], axis=1), axis=2).sum(axis=1)
        else:
            o["edge_px"][:] = np.nan
        ok = o["status"] == "ok"
        for metric in ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "perimeter_px"):
            m[metric][~ok] = np.nan
    return out


def half_areas(cleaned, masks, origins, n_angles=128, names=("half_area",), *, level=0.5, peak_pixels=4.0,
               outlines=True):
    """The half_area family on an (n, h, w) stack of neighbour-removed cells: for each name of
    `names` the oracle's measurement dict with the reference's metrics (local_level, threshold,
    mean_signal beside the geometry)."""
    specs = [{"name": name, "level": level, "background": HALF_AREA[name][0],
              "peak_pixels": peak_pixels if HALF_AREA[name][1] else None, "cuts": None} for name in names]
    return areas(cleaned, masks, origins, n_angles, specs, outlines=outlines)


# ---------------------------------------------------------------------------- the tail family
# subpx/_cpu/invariant_cd.py: _wide_cells 878-964 (CPU branch) and measure_invariant's tail branch
# 1009-1068: each reported hole on a square window of half-width ceil(tail_window * pitch) around its
# rounded fitted centre, holding its own share of the light, measured by the area methods with a low
# threshold.

TAIL_AREA = {"tail_area": "median", "tail_area_norm": "zero", "edge_area": "edge", "foot_area": "foot",
             "foot_area_ratio": "given"}


def wide_cells(signal, state, masks, origins, report, pitch, radius_pitches):
    """(cells as float32, inside the image, level pixels, own territory, window origins): the image
    minus the background map, each pixel shared among the holes in proportion to their models (own
    model / (model image + 1e-3 x the median amplitude)); territory = closer to the hole than to its
    8 nearest modelled holes; level pixels = the farthest tenth (at least 4) of the territory."""
    from scipy.spatial import cKDTree

    from .deblend import render_radius

    n_all, h, w = masks.shape
    cap = int(max(h, w))
    params = np.asarray(state.params, dtype=float).copy()
    params[:, 1:3] += origins
    fallback = origins + np.array([(w - 1) / 2, (h - 1) / 2])
    centers_all = np.where(np.isfinite(params[:, 1:3]), params[:, 1:3], fallback)
    rows_rep = np.arange(n_all)[report]
    centers = centers_all[rows_rep]
    radius = int(np.ceil(radius_pitches * pitch))
    size = 2 * radius + 1
    win_origins = np.rint(centers).astype(np.int64) - radius
    n = len(rows_rep)
    if not n:
        shape = (0, size, size)
        return (np.empty(shape, np.float32), np.empty(shape, bool), np.empty(shape, bool), np.empty(shape, bool),
                win_origins.astype(float))
    k = min(9, n_all)
    neighbours = cKDTree(centers_all).query(centers, k=k)[1].reshape(n, k)
    neighbours[:, 0] = rows_rep
    data = signal - state.background_map
    model = state.model_image
    good_amp = params[np.isfinite(params).all(axis=1), 0]
    floor = 1e-3 * float(np.median(good_amp)) if good_amp.size else 1e-12
    height, width = signal.shape
    offsets = np.arange(size)
    o = win_origins
    ys = o[:, 1, None] + offsets[None]
    xs = o[:, 0, None] + offsets[None]
    inside = ((ys >= 0) & (ys < height))[:, :, None] & ((xs >= 0) & (xs < width))[:, None, :]
    pick = (np.clip(ys, 0, height - 1)[:, :, None], np.clip(xs, 0, width - 1)[:, None, :])
    win, total = data[pick], model[pick]
    gp = params[rows_rep]
    good = np.isfinite(gp).all(axis=1)
    gp = np.where(good[:, None], gp, 0.0)
    render = render_radius(np.where(np.isfinite(params[rows_rep]), params[rows_rep], 0.0), cap)
    gx = xs[:, None, :].astype(float)
    gy = ys[:, :, None].astype(float)
    dx = gx - gp[:, 1, None, None]
    dy = gy - gp[:, 2, None, None]
    a = np.exp(gp[:, 3, None, None]) * dx + gp[:, 4, None, None] * dy
    b = np.exp(gp[:, 5, None, None]) * dy
    box = (np.abs(dx) <= render[:, None, None]) & (np.abs(dy) <= render[:, None, None]) & good[:, None, None]
    own = np.where(box, gp[:, 0, None, None] * np.exp(-0.5 * (a * a + b * b)), 0.0)
    near = centers_all[neighbours]
    dist = np.sqrt((gx[:, None] - near[:, :, 0, None, None]) ** 2 + (gy[:, None] - near[:, :, 1, None, None]) ** 2)
    mine = dist[:, 0] <= dist[:, 1:].min(axis=1) if k > 1 else np.ones_like(dist[:, 0], dtype=bool)
    own_area = inside & mine
    far = np.sort(np.where(own_area, dist[:, 0], -np.inf).reshape(n, -1), axis=1)[:, ::-1]
    count = own_area.reshape(n, -1).sum(axis=1)
    keep = np.clip(np.maximum(count // 10, 4), 1, far.shape[1]) - 1
    level = own_area & (dist[:, 0] >= far[np.arange(n), keep][:, None, None])
    cells = np.where(inside, win * own / (total + floor), 0.0).astype(np.float32)
    return cells, inside, level, own_area, win_origins.astype(float)


def median_pitch(state, origins):
    """The median nearest-neighbour distance of the fitted centres (measure_invariant's default pitch)."""
    from scipy.spatial import cKDTree

    centers = np.asarray(state.params)[:, 1:3] + origins
    centers = centers[np.isfinite(centers).all(axis=1)]
    return float(np.median(cKDTree(centers).query(centers, k=2)[0][:, 1])) if len(centers) > 1 else None


def tail_areas(signal, state, masks, origins, report, n_angles=128, names=("tail_area",), *, level=0.2,
               peak_pixels=4.0, window=1.2, pitch=None, outlines=True):
    """The tail family for the reported holes of a converged deblend state: per name the oracle's
    measurement dict (center_local relative to the hole's own cell), plus "_info" with the window
    size in pixels and foot_area_ratio's ratio."""
    masks = np.asarray(masks, dtype=bool)
    origins = np.asarray(origins, dtype=np.float64).reshape(-1, 2)
    if pitch is None or not np.isfinite(pitch):
        pitch = median_pitch(state, origins)
        if pitch is None:
            pitch = float(max(masks.shape[1:]))
    cells, inside, level_masks, territory, win_origins = wide_cells(signal, state, masks, origins, report, pitch,
                                                                    window)
    first = [name for name in names if name != "foot_area_ratio"]
    if "foot_area_ratio" in names and "foot_area" not in first:
        first.append("foot_area")
    specs = [{"name": name, "level": level, "background": TAIL_AREA[name], "peak_pixels": peak_pixels, "cuts": None}
             for name in first]
    found = areas(cells, inside, win_origins, n_angles, specs, level_masks=level_masks, zone_masks=territory,
                  outlines=outlines)
    info = {"tail_window_px": int(cells.shape[1])}
    if "foot_area_ratio" in names:
        foot = found["foot_area"]
        steepest = foot["metrics"]["steepest_level"]
        valid = foot["status"] == "ok"
        ratio = float(np.nanmedian((foot["metrics"]["threshold"] / steepest)[valid])) if valid.any() else np.nan
        info["foot_ratio"] = ratio
        found.update(areas(cells, inside, win_origins, n_angles,
                           [{"name": "foot_area_ratio", "level": level, "background": "given",
                             "peak_pixels": peak_pixels, "cuts": ratio * steepest}],
                           level_masks=level_masks, zone_masks=territory, outlines=outlines))
    rep_origins = origins[np.arange(len(origins))[report]]
    out = {}
    for name in names:
        o = found[name]
        local = o["centers"] - rep_origins
        o["center_local"] = np.where(np.isfinite(local), local, np.nan)
        out[name] = o
    out["_info"] = info
    return out
