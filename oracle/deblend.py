"""Oracle: deblending (background map + one Gaussian per hole) — CPU restatement, test infrastructure.

Follows subpx/_cpu/deblend.py: the model and its Jacobian (48-71), render_models (87-107), windows /
clean_cells (118-149), initial_params (152-171), fit_gaussians_batch (174-254), sigma_caps (257-259),
fit_status (262-277), _tile_medians / _upsample_tiles / _tile_centers (280-320), background_tiles
(346-393), auto_tile (396-403), deblend (421-522) and revise_seeds (525-567), over the same numerical
primitives (NumPy, scipy.ndimage, scipy.spatial).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FWHM_K = float(np.sqrt(2 * np.log(2)))
SIGMA_MIN = 0.5
RENDER_SIGMAS = 4.0


@dataclass
class State:
    background_map: np.ndarray
    model_image: np.ndarray
    params: np.ndarray
    status: np.ndarray
    cleaned: np.ndarray
    tile_px: int
    iterations: int
    background_info: dict
    converged: bool = False


def precision(params):
    e1, u2, e3 = np.exp(params[:, 3]), params[:, 4], np.exp(params[:, 5])
    m = np.empty((len(params), 2, 2))
    m[:, 0, 0] = e1 * e1
    m[:, 0, 1] = m[:, 1, 0] = e1 * u2
    m[:, 1, 1] = u2 * u2 + e3 * e3
    return m


def sigma_major(params):
    if len(params) == 0:
        return np.zeros(0)
    smallest = np.linalg.eigvalsh(precision(params))[:, 0]
    return 1 / np.sqrt(np.maximum(smallest, 1e-300))


def gaussian(params, dx, dy):
    """Model values plus the factors the Jacobian reuses, for (N, K) offsets."""
    e1 = np.exp(params[:, 3])[:, None]
    u2 = params[:, 4][:, None]
    e3 = np.exp(params[:, 5])[:, None]
    a = e1 * dx + u2 * dy
    b = e3 * dy
    shape = np.exp(-0.5 * (a * a + b * b))
    return params[:, 0][:, None] * shape, shape, a, b, e1, u2, e3


def render_radius(params, cap):
    return np.clip(np.ceil(RENDER_SIGMAS * sigma_major(params)), 2, cap)


def truncated(params_global, gx, gy, radius):
    dx = gx - params_global[:, 1][:, None]
    dy = gy - params_global[:, 2][:, None]
    vals = gaussian(params_global, dx, dy)[0]
    inside = (np.abs(dx) <= radius[:, None]) & (np.abs(dy) <= radius[:, None])
    return np.where(inside, vals, 0.0)


def render(params_global, shape, radius_cap):
    """Sum of every hole's truncated Gaussian (global centres) on an (H, W) image."""
    h, w = shape
    out = np.zeros(h * w)
    if len(params_global) == 0:
        return out.reshape(shape)
    radius = render_radius(params_global, radius_cap)
    rmax = int(radius.max())
    off = np.arange(-rmax, rmax + 1)
    chunk = max(1, 2_000_000 // len(off) ** 2)
    for s in range(0, len(params_global), chunk):
        p = params_global[s:s + chunk]
        ix = np.floor(p[:, 1]).astype(np.int64)[:, None, None] + off[None, None, :]
        iy = np.floor(p[:, 2]).astype(np.int64)[:, None, None] + off[None, :, None]
        ix, iy = (a.reshape(len(p), -1) for a in np.broadcast_arrays(ix, iy))
        vals = truncated(p, ix.astype(float), iy.astype(float), radius[s:s + chunk])
        ok = (ix >= 0) & (ix < w) & (iy >= 0) & (iy < h) & (vals != 0)
        out += np.bincount((iy * w + ix)[ok], weights=vals[ok], minlength=h * w)
    return out.reshape(shape)


def windows(image, origins, shape):
    h, w = image.shape
    ys = origins[:, 1, None] + np.arange(shape[0])[None]
    xs = origins[:, 0, None] + np.arange(shape[1])[None]
    inside = ((ys >= 0) & (ys < h))[:, :, None] & ((xs >= 0) & (xs < w))[:, None, :]
    vals = image[np.clip(ys, 0, h - 1)[:, :, None], np.clip(xs, 0, w - 1)[:, None, :]]
    return np.where(inside, vals, 0.0)


def grids(origins, shape):
    yy, xx = np.indices(shape, dtype=float)
    gx = (origins[:, 0, None, None] + xx[None]).reshape(len(origins), -1)
    gy = (origins[:, 1, None, None] + yy[None]).reshape(len(origins), -1)
    return gx, gy


def clean(raw, background, model, params_global, masks, origins, radius_cap, grid):
    shape = masks.shape[1:]
    own = truncated(params_global, *grid, render_radius(params_global, radius_cap)).reshape(masks.shape)
    return np.where(masks, raw - windows(background, origins, shape) - (windows(model, origins, shape) - own), 0.0)


def initial_params(data, masks, seeds_local):
    n = len(data)
    p = np.zeros((n, 6))
    if n == 0:
        return p
    peak = np.where(masks, data, -np.inf).reshape(n, -1).max(axis=1)
    wgt = np.where(masks & (data > 0.2 * peak[:, None, None]), data, 0.0)
    yy, xx = np.indices(data.shape[1:], dtype=float)
    total = np.maximum(wgt.sum(axis=(1, 2)), 1e-300)
    dx = xx[None] - seeds_local[:, 0, None, None]
    dy = yy[None] - seeds_local[:, 1, None, None]
    var = ((wgt * (dx * dx + dy * dy)).sum(axis=(1, 2)) / total) / 2
    sig = np.sqrt(np.clip(var, 0.25, None))
    p[:, 0] = np.maximum(peak, 1e-12)
    p[:, 1:3] = seeds_local
    p[:, 3] = p[:, 5] = -np.log(sig)
    return p


def sigma_caps(masks):
    return np.maximum(1.0, np.sqrt(masks.reshape(len(masks), -1).sum(axis=1) / np.pi))


def fit_status(p, masks, cap, status):
    h, w = masks.shape[1:]
    bad = ~np.isfinite(p).all(axis=1)
    sig = np.full(len(p), np.nan)
    sig[~bad] = sigma_major(p[~bad])
    status[bad] = "fit_diverged"
    status[~bad & ((p[:, 0] <= 0) | (sig >= 0.999 * cap))] = "non_gaussian_fit"
    c = np.where(np.isfinite(p[:, 1:3]), p[:, 1:3], 0.0)
    iy = np.round(c[:, 1]).astype(int).clip(0, h - 1)
    ix = np.round(c[:, 0]).astype(int).clip(0, w - 1)
    inside = (p[:, 1] >= -0.5) & (p[:, 1] <= w - 0.5) & (p[:, 2] >= -0.5) & (p[:, 2] <= h - 0.5)
    inside &= masks[np.arange(len(p)), iy, ix]
    status[(status == "ok") & ~inside] = "center_outside_cell"


def fit_batch(data, masks, init, max_iter=30):
    """Levenberg-Marquardt fit of one Gaussian per cell, all cells at once."""
    n, h, w = data.shape
    params = init.astype(np.float64).copy()
    status = np.full(n, "ok", dtype="U32")
    if n == 0:
        return params, status
    yy, xx = np.indices((h, w), dtype=float)
    xx, yy = xx.ravel(), yy.ravel()
    caps = sigma_caps(masks)
    chunk = max(1, 2_000_000 // (h * w * 6))
    for s in range(0, n, chunk):
        sl = slice(s, s + chunk)
        d = data[sl].reshape(-1, h * w)
        wt = masks[sl].reshape(-1, h * w).astype(float)
        p = params[sl]
        lam = np.full(len(p), 1e-3)
        cap = caps[sl]
        amp_cap = 3 * np.maximum(np.abs(np.where(wt > 0, d, 0)).max(axis=1), 1e-12)

        def cost(q, rows):
            r = d[rows] - gaussian(q, xx[None] - q[:, 1, None], yy[None] - q[:, 2, None])[0]
            return (wt[rows] * r * r).sum(axis=1)

        c = cost(p, slice(None))
        active = np.isfinite(c)
        for _ in range(max_iter):
            if not active.any():
                break
            q = p[active]
            dx, dy = xx[None] - q[:, 1, None], yy[None] - q[:, 2, None]
            model, shp, a, b, e1, u2, e3 = gaussian(q, dx, dy)
            half = -0.5 * model
            jac = np.stack((shp, half * (-2 * a * e1), half * (-2 * a * u2 - 2 * b * e3), half * (2 * a * e1 * dx),
                            half * (2 * a * dy), half * (2 * b * e3 * dy)), axis=2)
            r = d[active] - model
            jw = jac * wt[active][:, :, None]
            normal = np.einsum("nki,nkj->nij", jw, jac)
            grad = np.einsum("nki,nk->ni", jw, r)
            diag = np.einsum("nii->ni", normal)
            damped = normal + (lam[active][:, None] * diag + 1e-12)[:, :, None] * np.eye(6)
            try:
                step = np.linalg.solve(damped, grad[:, :, None])[:, :, 0]
            except np.linalg.LinAlgError:
                step = np.stack([np.linalg.lstsq(m, g, rcond=None)[0] for m, g in zip(damped, grad)])
            trial = q + step
            lo = -np.log(cap[active])
            trial[:, 0] = np.clip(trial[:, 0], 0.0, amp_cap[active])
            trial[:, 3] = np.clip(trial[:, 3], lo, -np.log(SIGMA_MIN))
            trial[:, 5] = np.clip(trial[:, 5], lo, -np.log(SIGMA_MIN))
            nc = cost(trial, active)
            better = np.isfinite(nc) & (nc <= c[active])
            idx = np.flatnonzero(active)
            p[idx[better]] = trial[better]
            lam[idx[better]] /= 3
            lam[idx[~better]] *= 4
            small = np.abs(step).max(axis=1) < 1e-7
            done = (better & (c[active] - nc <= 1e-12 * np.maximum(c[active], 1e-300))) | small
            c[idx[better]] = nc[better]
            active[idx[done | (lam[idx] > 1e12)]] = False
        params[sl] = p
        fit_status(p, masks[sl], cap, status[sl])
    return params, status


def tile_centers(tile, shape):
    h, w = shape
    yc = np.array([(j * tile + min((j + 1) * tile, h) - 1) / 2 for j in range(-(-h // tile))])
    xc = np.array([(i * tile + min((i + 1) * tile, w) - 1) / 2 for i in range(-(-w // tile))])
    return yc, xc


def tile_medians(values, usable, tile):
    h, w = values.shape
    ny, nx = -(-h // tile), -(-w // tile)
    padded = np.full((ny * tile, nx * tile), np.nan)
    padded[:h, :w] = np.where(usable, values, np.nan)
    blocks = padded.reshape(ny, tile, nx, tile).transpose(0, 2, 1, 3).reshape(ny, nx, tile * tile)
    counts = np.isfinite(blocks).sum(axis=2)
    med = np.full((ny, nx), np.nan)
    has = counts > 0
    med[has] = np.nanmedian(blocks[has], axis=1)
    return med, counts


def upsample(medians, tile, shape):
    h, w = shape
    ny, _ = medians.shape
    yc, xc = tile_centers(tile, shape)
    rows = np.stack([np.interp(np.arange(w), xc, medians[j]) for j in range(ny)])
    if ny == 1:
        return np.repeat(rows, h, axis=0)
    y = np.arange(h, dtype=float)
    j1 = np.clip(np.searchsorted(yc, y), 1, ny - 1)
    t = np.clip((y - yc[j1 - 1]) / (yc[j1] - yc[j1 - 1]), 0, 1)[:, None]
    return (1 - t) * rows[j1 - 1] + t * rows[j1]


def background_tiles(residual, free, usable, tile):
    from scipy.interpolate import LinearNDInterpolator
    from scipy.spatial import Delaunay, cKDTree

    shape = residual.shape
    free_med, free_count = tile_medians(residual, free & usable, tile)
    measured = free_count >= max(16, int(0.1 * tile * tile))
    info = {"tiles": int(measured.size), "measured_tiles": int(measured.sum())}
    if measured.all():
        med, info["source"] = free_med, "measured"
    elif measured.any():
        yc, xc = tile_centers(tile, shape)
        grid = np.stack(np.meshgrid(yc, xc, indexing="ij"), axis=-1)
        known, vals = grid[measured], free_med[measured]
        try:
            tri = Delaunay(known) if len(vals) >= 3 else None
        except Exception:
            tri = None
        med = free_med.copy()
        missing = ~measured
        med[missing] = np.nan
        if tri is not None:
            med[missing] = LinearNDInterpolator(tri, vals)(grid[missing])
        still = missing & np.isnan(med)
        med[still] = vals[cKDTree(known).query(grid[still])[1]]
        info["source"] = "interpolated"
    else:
        med, _ = tile_medians(residual, usable, tile)
        info["source"] = "inferred"
        if np.isnan(med).all():
            return None, info
        med = np.where(np.isnan(med), np.nanmedian(med), med)
    info["tile_medians"] = med
    return med, info


def auto_tile(seeds, shape):
    from scipy.spatial import cKDTree

    if len(seeds) < 2:
        return int(max(shape)), float("nan")
    pitch = float(np.median(cKDTree(seeds).query(seeds, k=2)[0][:, 1]))
    return int(np.clip(round(4 * pitch), 16, max(shape))), pitch


def deblend(image, seeds, masks, origins, *, iterations=30, tile=None, exclude=None, background_level=None,
            free_fraction=0.05, free_distance_fwhm=1.25, relaxation=0.6, tolerance=1e-3, max_iter=30, init=None):
    from scipy.ndimage import binary_erosion, distance_transform_edt

    image = np.asarray(image, dtype=np.float64)
    shape = image.shape
    seeds = np.asarray(seeds, float).reshape(-1, 2)
    n = len(seeds)
    origins = np.asarray(origins, dtype=np.int64).reshape(-1, 2)
    tile = int(auto_tile(seeds, shape)[0] if tile is None else tile)
    usable = np.ones(shape, bool) if exclude is None else ~exclude
    seed_px = np.ones(shape, bool)
    if n:
        seed_px[np.clip(np.rint(seeds[:, 1]).astype(int), 0, shape[0] - 1),
                np.clip(np.rint(seeds[:, 0]).astype(int), 0, shape[1] - 1)] = False
    dist = distance_transform_edt(seed_px) if n else np.full(shape, np.inf)

    def background_of(residual, model, p, st):
        if background_level is not None:
            return np.full(shape, float(background_level)), {"source": "fixed"}
        good = (st == "ok") & (p[:, 0] > 0)
        amp = float(np.median(p[good, 0])) if good.any() else 1.0
        fwhm = float(np.median(2 * FWHM_K * sigma_major(p[good]))) if good.any() else 0.0
        free = (model < free_fraction * amp) & (dist >= free_distance_fwhm * fwhm)
        med, info = background_tiles(residual, free, usable, tile)
        if med is None:
            return np.full(shape, float(np.median(residual))), info
        return upsample(med, tile, shape), info

    if n == 0:
        bg, info = background_of(image, np.zeros(shape), np.zeros((0, 6)), np.zeros(0, "U32"))
        return State(bg, np.zeros(shape), np.zeros((0, 6)), np.zeros(0, "U32"), np.zeros(masks.shape), tile, 0,
                     info, False)
    roi = masks.shape[1:]
    raw = windows(image, origins, roi)
    grid = grids(origins, roi)
    cap_r = int(max(roi))
    caps = sigma_caps(masks)
    if init is None:
        border = masks & ~binary_erosion(masks, structure=np.ones((1, 3, 3)), border_value=0)
        bg0 = np.array([np.percentile(r[b], 10) if b.any() else 0.0 for r, b in zip(raw, border)])
        if background_level is not None:
            bg0[:] = background_level
        data = np.where(masks, raw - bg0[:, None, None], 0.0)
        params, status = fit_batch(data, masks, initial_params(data, masks, seeds - origins), max_iter)
    else:
        params, status = np.asarray(init, dtype=np.float64).copy(), np.full(n, "ok", dtype="U32")
        fit_status(params, masks, caps, status)

    def glob(p):
        g = p.copy()
        g[:, 1:3] += origins
        return g

    model = render(glob(params), shape, cap_r)
    used, converged = 0, False
    for used in range(1, int(iterations) + 1):
        bg, info = background_of(image - model, model, params, status)
        fitted, status = fit_batch(clean(raw, bg, model, glob(params), masks, origins, cap_r, grid), masks, params,
                                   max_iter)
        step = np.where(np.isfinite(fitted), fitted - params, 0.0)
        params = params + relaxation * step
        status = np.full(n, "ok", dtype="U32")
        fit_status(params, masks, caps, status)
        model = render(glob(params), shape, cap_r)
        ok = (status == "ok") & np.isfinite(fitted).all(axis=1)
        if not ok.any():
            break
        if np.percentile(np.abs(step[ok][:, 1:]).max(axis=1), 99) < tolerance:
            converged = True
            break
    bg, info = background_of(image - model, model, params, status)
    return State(bg, model, params, status, clean(raw, bg, model, glob(params), masks, origins, cap_r, grid), tile,
                 used, info, converged)


def revise_seeds(signal, state, seeds, pitch, *, drop_fraction=0.3, add_fraction=0.5, exclude=None):
    from scipy.ndimage import gaussian_filter, maximum_filter
    from scipy.spatial import cKDTree

    p = state.params
    finite = np.isfinite(p).all(axis=1)
    good = finite & (state.status == "ok") & (p[:, 0] > 0)
    if not good.any():
        return np.zeros(len(p), bool), np.zeros((0, 2))
    ref = float(np.median(p[good, 0]))
    drop = ~finite | (p[:, 0] < drop_fraction * ref)
    resid = signal - state.background_map - state.model_image
    smooth = gaussian_filter(resid, max(0.5, 0.1 * pitch), mode="nearest")
    rad = max(1, int(np.floor(0.5 * pitch)))
    peaks = (smooth == maximum_filter(smooth, size=2 * rad + 1, mode="nearest")) & (smooth > add_fraction * ref)
    ys, xs = np.nonzero(peaks)
    if exclude is not None:
        keep = ~np.asarray(exclude, bool)[ys, xs]
        ys, xs = ys[keep], xs[keep]
    new = np.column_stack((xs, ys)).astype(float)
    kept = np.asarray(seeds, float)[~drop]
    if len(new) and len(kept):
        new = new[cKDTree(kept).query(new)[0] > 0.5 * pitch]
    return drop, new


def estimate_pitch(signal, *, max_size=1024):
    """Lattice pitch from the first ring of the radially averaged autocorrelation of a centred crop
    (subpx/_cpu/deblend.py:570-590): zero-padded FFT autocorrelation, integer radius bins
    (np.rint of the distance to the zero lag) up to half the crop, first local maximum k >= 2 of
    the bin means refined by a parabola through its neighbours."""
    h, w = signal.shape
    y0, x0 = max(0, (h - max_size) // 2), max(0, (w - max_size) // 2)
    crop = np.asarray(signal[y0:y0 + max_size, x0:x0 + max_size], dtype=np.float64)
    crop = crop - crop.mean()
    size = (2 * crop.shape[0], 2 * crop.shape[1])
    auto = np.fft.fftshift(np.fft.irfft2(np.abs(np.fft.rfft2(crop, s=size)) ** 2, s=size))
    cy, cx = np.array(auto.shape) // 2
    yy, xx = np.indices(auto.shape)
    bins = np.rint(np.hypot(yy - cy, xx - cx)).astype(int)
    keep = bins <= int(min(crop.shape) // 2)
    prof = np.bincount(bins[keep], weights=auto[keep]) / np.maximum(np.bincount(bins[keep]), 1)
    for k in range(2, len(prof) - 1):
        if prof[k] > prof[k - 1] and prof[k] >= prof[k + 1] and prof[k] > 0:
            den = prof[k - 1] - 2 * prof[k] + prof[k + 1]
            return float(k + (0.5 * (prof[k - 1] - prof[k + 1]) / den if den < 0 else 0.0))
    raise ValueError("could not estimate the hole pitch; pass peak_min_distance explicitly")


def detect_peaks(signal, *, min_distance=None, smooth_sigma=None, threshold=0.25):
    """Local-maximum seeds of a dense array (subpx/_cpu/deblend.py:593-630): maxima of the smoothed
    signal over a (2 floor(min_distance) + 1)^2 window whose prominence over the minimum of a
    (2 ceil(pitch) + 1)^2 window is positive and at least `threshold` x its 90th percentile over
    all maxima, in row-major order, each moved by the clipped parabola vertex of its row and column
    neighbours. Returns (seeds_xy, pitch)."""
    from scipy.ndimage import gaussian_filter, maximum_filter, minimum_filter

    signal = np.asarray(signal, dtype=np.float64)
    pitch = 2.0 * float(min_distance) if min_distance is not None else estimate_pitch(signal)
    if min_distance is None:
        min_distance = 0.5 * pitch
    if smooth_sigma is None:
        smooth_sigma = max(0.5, 0.1 * pitch)
    smooth = gaussian_filter(signal, smooth_sigma, mode="nearest")
    rad = max(1, int(np.floor(min_distance)))
    is_max = smooth == maximum_filter(smooth, size=2 * rad + 1, mode="nearest")
    prom = smooth - minimum_filter(smooth, size=2 * int(np.ceil(pitch)) + 1, mode="nearest")
    ys, xs = np.nonzero(is_max & (prom > 0))
    if len(xs) == 0:
        return np.zeros((0, 2)), pitch
    pv = prom[ys, xs]
    keep = pv >= threshold * np.percentile(pv, 90)
    ys, xs = ys[keep], xs[keep]
    h, w = signal.shape
    sub = np.column_stack((xs, ys)).astype(float)
    for axis, (dy, dx) in enumerate(((0, 1), (1, 0))):
        ok = (ys - dy >= 0) & (ys + dy < h) & (xs - dx >= 0) & (xs + dx < w)
        left = smooth[np.clip(ys - dy, 0, h - 1), np.clip(xs - dx, 0, w - 1)]
        mid = smooth[ys, xs]
        right = smooth[np.clip(ys + dy, 0, h - 1), np.clip(xs + dx, 0, w - 1)]
        curv = left - 2 * mid + right
        delta = np.where(ok & (curv < 0), 0.5 * (left - right) / np.where(curv < 0, curv, -1), 0.0)
        sub[:, axis] += np.clip(delta, -0.5, 0.5)
    return sub, pitch


def initial_fits(image, seeds, masks, origins, *, background_level=None, max_iter=30):
    """The initial fits that start deblend (subpx/_cpu/deblend.py:452-480): per cell the 10th
    percentile of its border pixels as background (or the given level), initial_params, LM and
    fit_status. Returns (params, status) in cell-local coordinates."""
    from scipy.ndimage import binary_erosion

    image = np.asarray(image, dtype=np.float64)
    seeds = np.asarray(seeds, float).reshape(-1, 2)
    origins = np.asarray(origins, dtype=np.int64).reshape(-1, 2)
    raw = windows(image, origins, masks.shape[1:])
    border = masks & ~binary_erosion(masks, structure=np.ones((1, 3, 3)), border_value=0)
    bg0 = np.array([np.percentile(r[b], 10) if b.any() else 0.0 for r, b in zip(raw, border)])
    if background_level is not None:
        bg0[:] = background_level
    data = np.where(masks, raw - bg0[:, None, None], 0.0)
    return fit_batch(data, masks, initial_params(data, masks, seeds - origins), max_iter)
