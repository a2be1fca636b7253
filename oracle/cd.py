"""Oracle: measure_cds with the model background — CPU restatement, test infrastructure.

Follows subpx/cd.py:424-784 (_measure_cds, background="model", seeds="threshold") and
subpx/_cpu/cd.py (_inside 19-25, _geometry 35-47, _logquad 50-89, _half_max_ellipse 92-107,
_ellipse_geometry 131-141, gaussian_method 144-192, _radial_profiles 195-217, _radial_contour 220-264,
measure_cells 267-322), with the same primitives (numpy.linalg, scipy.ndimage.map_coordinates,
binary_erosion / binary_dilation). Returns plain dicts of arrays.
"""

from __future__ import annotations

import numpy as np

from . import deblend as odb
from . import segment as osg
from . import voronoi as ov

K = float(np.sqrt(2 * np.log(2)))
GEOMETRY = ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "perimeter_px")
FIT = ("sigma_major_px", "sigma_minor_px", "fwhm_major_px", "fwhm_minor_px", "angle_deg", "log_fit_rmse")


def _inside(points, mask):
    from scipy.ndimage import map_coordinates

    return map_coordinates(mask.astype(float), points.T[::-1], order=1, mode="constant", cval=0,
                           prefilter=False) >= 1 - 1e-8


def _polygon(contour):
    v = contour - contour[0]
    area = abs(np.sum(v[:-1, 0] * v[1:, 1] - v[1:, 0] * v[:-1, 1])) / 2
    return {"area_px2": float(area), "cd_equivalent_px": float(2 * np.sqrt(area / np.pi)),
            "cd_x_px": float(np.ptp(contour[:, 0])), "cd_y_px": float(np.ptp(contour[:, 1])),
            "perimeter_px": float(np.linalg.norm(np.diff(contour, axis=0), axis=1).sum())}


def _ellipse(center, eigenvalues, axes, angles):
    sigma = 1 / np.sqrt(eigenvalues)
    contour = None
    if angles is not None:
        circle = np.column_stack((np.cos(angles), np.sin(angles)))
        contour = center + (circle * (K * sigma)) @ axes.T
        contour = np.vstack((contour, contour[0]))
    cov = (axes * (sigma * sigma)) @ axes.T
    fit = dict(sigma_major_px=float(sigma[0]), sigma_minor_px=float(sigma[1]), fwhm_major_px=float(2 * K * sigma[0]),
               fwhm_minor_px=float(2 * K * sigma[1]),
               angle_deg=float(np.degrees(np.arctan2(axes[1, 0], axes[0, 0])) % 180))
    return contour, sigma, cov, fit


def _ellipse_geometry(contour, sigma, cov):
    g = _polygon(contour) if contour is not None else {"perimeter_px": float("nan")}
    area = float(np.pi * K ** 2 * np.prod(sigma))
    g.update(area_px2=area, cd_equivalent_px=float(2 * np.sqrt(area / np.pi)),
             cd_x_px=float(2 * K * np.sqrt(cov[0, 0])), cd_y_px=float(2 * K * np.sqrt(cov[1, 1])))
    return g


def _logquad(roi, mask, seed, angles, fit_fraction):
    signal = roi
    peak = float(signal[mask].max())
    missing = np.full((len(angles) + 1, 2), np.nan)
    extra = {"background": 0.0, "peak_signal": peak}
    if peak <= 0:
        return seed, missing, extra, "no_signal", None
    fm = mask & (signal > fit_fraction * peak)
    yy, xx = np.nonzero(fm)
    if len(xx) < 6:
        return seed, missing, extra, "insufficient_fit_pixels", None
    x, y = xx - seed[0], yy - seed[1]
    design = np.column_stack((x * x, y * y, x * y, x, y, np.ones(len(x))))
    z = np.log(signal[fm])
    wgt = signal[fm] / peak
    coef, _, rank, _ = np.linalg.lstsq(design * wgt[:, None], z * wgt, rcond=None)
    if rank < 6:
        return seed, missing, extra, "singular_fit", None
    a, b, c, d, e, _ = coef
    prec = -np.array([[2 * a, c], [c, 2 * b]])
    ev, ax = np.linalg.eigh(prec)
    if ev[0] <= 1e-10 or ev[-1] / ev[0] > 1e8:
        return seed, missing, extra, "non_gaussian_fit", None
    center = seed + np.linalg.solve(prec, [d, e])
    contour, sigma, cov, fit = _ellipse(center, ev, ax, angles)
    extra.update(fit, log_fit_rmse=float(np.sqrt(np.average((design @ coef - z) ** 2, weights=wgt ** 2))))
    if not _inside(np.vstack((center, contour)), mask).all():
        return center, contour, extra, "contour_outside_cell", (ev, ax)
    extra.update(_ellipse_geometry(contour, sigma, cov))
    return center, contour, extra, "ok", (ev, ax)


def _radial(roi, mask, angles, step, smooth_sigma=0.0):
    from scipy.ndimage import binary_erosion, gaussian_filter, map_coordinates

    signal = np.where(mask, roi, 0)
    wgt = np.where(mask & (signal > 0.1 * signal.max()), signal, 0)
    yy, xx = np.indices(roi.shape)
    center = np.array([(wgt * xx).sum(), (wgt * yy).sum()]) / wgt.sum()
    if smooth_sigma > 0:
        # Mask-normalised smoothing (subpx/_cpu/cd.py:206-208); the centre comes from the raw signal.
        support = gaussian_filter(mask.astype(float), smooth_sigma, mode="constant")
        signal = gaussian_filter(signal, smooth_sigma, mode="constant") / np.maximum(support, 1e-12)
    radii = np.arange(0, np.hypot(*roi.shape) + step, step)
    dirs = np.column_stack((np.cos(angles), np.sin(angles)))
    pts = center + dirs[:, None, :] * radii[None, :, None]
    prof = map_coordinates(signal, pts.transpose(2, 0, 1)[::-1], order=3, mode="nearest")
    valid = _inside(pts.reshape(-1, 2), binary_erosion(mask, border_value=0)).reshape(prof.shape)
    valid = np.logical_and.accumulate(valid, axis=1)
    return center, radii, prof, valid


def _radial_edges(method, center, radii, prof, valid, angles):
    n = len(angles)
    edge = np.full(n, np.nan)
    peak = float(prof[0, 0])
    extra = {"background": 0.0, "peak_signal": peak, "ray_coverage": 0.0}
    if peak > 0:
        if method == "halfmax":
            cross = (prof[:, :-1] >= peak / 2) & (prof[:, 1:] < peak / 2) & valid[:, :-1] & valid[:, 1:]
            found = cross.any(axis=1)
            ray = np.flatnonzero(found)
            j = np.argmax(cross[found], axis=1)
            frac = (prof[ray, j] - peak / 2) / (prof[ray, j] - prof[ray, j + 1])
            edge[found] = radii[j] + frac * (radii[1] - radii[0])
        else:
            step = radii[1] - radii[0]
            grad = -np.gradient(prof, step, axis=1)
            cand = np.zeros_like(valid)
            cand[:, 2:-2] = valid[:, :-4] & valid[:, 4:]
            cand &= radii[None, :] >= max(0.35, 2 * step)
            j = np.argmax(np.where(cand, grad, -np.inf), axis=1)
            ray = np.arange(n)
            jm, jp = np.maximum(j - 1, 0), np.minimum(j + 1, len(radii) - 1)
            left, mid, right = grad[ray, jm], grad[ray, j], grad[ray, jp]
            found = cand[ray, j] & cand[ray, jm] & cand[ray, jp] & (mid >= left) & (mid >= right) & (mid > 0.01 * peak)
            curv = left - 2 * mid + right
            found &= curv < -1e-12
            delta = np.zeros(n)
            delta[found] = 0.5 * (left[found] - right[found]) / curv[found]
            edge[found] = radii[j[found]] + np.clip(delta[found], -0.5, 0.5) * step
    pts = center + edge[:, None] * np.column_stack((np.cos(angles), np.sin(angles)))
    contour = np.vstack((pts, pts[0]))
    extra["ray_coverage"] = float(np.isfinite(edge).mean())
    if not np.isfinite(edge).all():
        return center, contour, extra, "incomplete_rays", edge
    extra.update(_polygon(contour))
    return center, contour, extra, "ok", edge


def _new_method(method, n, n_angles):
    names = GEOMETRY + ("background", "peak_signal") + (FIT if method == "logquad" else ("ray_coverage",))
    return {"centers": np.full((n, 2), np.nan), "contours": np.full((n, n_angles + 1, 2), np.nan),
            "status": np.full(n, "no_signal", dtype="U32"), "metrics": {m: np.full(n, np.nan) for m in names},
            "edge_px": np.full((n, n_angles), np.nan)}


def measure_cells(rois, masks, origins, seeds, *, methods, n_angles=128, radial_step=0.1, fit_fraction=0.2,
                  smooth_sigma=0.0):
    n = len(rois)
    angles = np.arange(n_angles) * (2 * np.pi / n_angles)
    res = {m: _new_method(m, n, n_angles) for m in methods}
    for i in range(n):
        roi, mask, origin, seed = rois[i], masks[i], origins[i], seeds[i]
        if mask.sum() < 6:
            for r in res.values():
                r["status"][i] = "insufficient_cell_pixels"
            continue
        if roi[mask].max() <= 0:
            continue
        radial = None
        for m, r in res.items():
            if m == "logquad":
                center, contour, met, st, _ = _logquad(roi, mask, seed - origin, angles, fit_fraction)
            else:
                if radial is None:
                    radial = _radial(roi, mask, angles, radial_step, smooth_sigma)
                center, contour, met, st, edge = _radial_edges(m, *radial, angles)
                r["edge_px"][i] = edge
            r["centers"][i] = center + origin
            r["contours"][i] = contour + origin
            r["status"][i] = st
            for k, v in met.items():
                r["metrics"][k][i] = v
    return res


def gaussian_method(params, status, cleaned, masks, origins, n_angles):
    n = len(params)
    angles = np.arange(n_angles) * (2 * np.pi / n_angles)
    names = GEOMETRY + ("background", "peak_signal") + FIT[:-1] + ("fit_rmse",)
    out = {"centers": np.full((n, 2), np.nan), "contours": np.full((n, n_angles + 1, 2), np.nan),
           "status": np.asarray(status, dtype="U32").copy(), "metrics": {m: np.full(n, np.nan) for m in names}}
    if n == 0:
        return out
    yy, xx = np.indices(cleaned.shape[1:], dtype=float)
    dx = xx.ravel()[None] - params[:, 1, None]
    dy = yy.ravel()[None] - params[:, 2, None]
    model = odb.gaussian(params, dx, dy)[0].reshape(cleaned.shape)
    resid = np.where(masks, cleaned - model, 0.0)
    rmse = np.sqrt((resid ** 2).sum(axis=(1, 2)) / np.maximum(masks.sum(axis=(1, 2)), 1))
    prec = odb.precision(params)
    for i in range(n):
        out["metrics"]["peak_signal"][i] = params[i, 0]
        out["metrics"]["fit_rmse"][i] = rmse[i]
        if not np.isfinite(params[i]).all():
            continue
        center = params[i, 1:3] + origins[i]
        out["centers"][i] = center
        ev, ax = np.linalg.eigh(prec[i])
        if ev[0] <= 1e-10:
            out["status"][i] = "non_gaussian_fit"
            continue
        contour, sigma, cov, fit = _ellipse(center, ev, ax, angles)
        out["contours"][i] = contour
        for k, v in fit.items():
            out["metrics"][k][i] = v
        if out["status"][i] == "ok":
            for k, v in _ellipse_geometry(contour, sigma, cov).items():
                out["metrics"][k][i] = v
    return out


def cell_stack(labels, rows, pad, shape):
    """Cell masks and origins of the rows' boxes (subpx/_gpu/cells.py:11-38)."""
    origins, sizes = ov.cell_boxes(rows, shape, pad)
    return ov.cell_masks(labels, origins, sizes), origins


def unmodelled(binary, labels, ids):
    from scipy.ndimage import binary_dilation

    modelled = np.zeros(int(labels.max(initial=0)) + 1, bool)
    ids = ids[(ids >= 0) & (ids < len(modelled))]
    modelled[ids] = True
    feats = binary & ~modelled[labels]
    return binary_dilation(feats, iterations=2)


def measure_cds(img, *, methods=("gaussian", "logquad", "gradient", "halfmax"), threshold="otsu", invert=False,
                area_min=3, area_max=50, pad=3, n_angles=128, radial_step=0.1, fit_fraction=0.2,
                deblend_iterations=30, deblend_tolerance=1e-3, background_level=None, seeds="threshold",
                peak_min_distance=None, smooth_sigma=0.0, tail_area_level=0.2, tail_window=1.2, psf_fwhm=None,
                nominal_cd=None, dark_level=0.0, flux_ratio_scale=None):
    """The model-background measure_cds pipeline, seeds from thresholded components or, with
    seeds="peaks", from the smoothed signal's maxima (subpx/cd.py:502-511)."""
    img = np.asarray(img)
    h, w = img.shape
    sign = -1.0 if invert else 1.0
    signal = img.astype(np.float64) * sign
    if seeds == "peaks":
        return _measure_peaks(img, signal, sign, methods=methods, pad=pad, n_angles=n_angles, radial_step=radial_step,
                              fit_fraction=fit_fraction, deblend_iterations=deblend_iterations,
                              deblend_tolerance=deblend_tolerance, background_level=background_level,
                              peak_min_distance=peak_min_distance, smooth_sigma=smooth_sigma,
                              tail_area_level=tail_area_level, tail_window=tail_window,
                              psf_fwhm=psf_fwhm, nominal_cd=nominal_cd, dark_level=sign * float(dark_level),
                              flux_ratio_scale=flux_ratio_scale)
    seg = img
    if img.dtype != np.uint8 and not (img.dtype == np.uint16 and threshold == "otsu"):
        g = img.astype(np.float64)
        span = float(g.max() - g.min())
        seg = np.rint((g - g.min()) * (255 / span)).astype(np.uint8) if span else np.zeros(img.shape, np.uint8)
    t = osg.otsu_threshold(seg) if threshold == "otsu" else osg.triangle_threshold(seg)
    binary = osg.binarize(seg, t, invert)
    num, labels, stats, cents = osg.label_components(binary, 8)
    x, y, bw, bh, area = stats[1:num].astype(np.int64).T
    keep = (area >= area_min) & (area <= area_max)
    oversized = np.zeros(num, bool)
    oversized[1:][area > area_max] = True
    oversized = oversized[labels] if oversized.any() else None
    inside = ~((x <= 0) | (y <= 0) | (x + bw >= w) | (y + bh >= h))
    rows = np.column_stack((x, y, bw, bh, cents[1:num])).astype(np.float64)[keep]
    ids = (np.flatnonzero(keep) + 1).astype(np.int32)
    interior = inside[keep]

    def build(rows_):
        seeds_ = rows_[:, 4:6].copy()
        lab_ = ov.voronoi_labels(seeds_, img.shape)
        masks_, origins_ = cell_stack(lab_, rows_, pad, img.shape)
        return seeds_, lab_, masks_, origins_

    seeds, cell_labels, masks, origins = build(rows)
    tile_px, pitch = odb.auto_tile(seeds, img.shape)
    return _deblend_and_measure(img, signal, sign, rows, ids, interior, np.zeros(len(rows), bool), pitch,
                                tile_px, unmodelled(binary, labels, ids), oversized, methods=methods, pad=pad,
                                n_angles=n_angles, radial_step=radial_step, fit_fraction=fit_fraction,
                                deblend_iterations=deblend_iterations, deblend_tolerance=deblend_tolerance,
                                background_level=background_level, smooth_sigma=smooth_sigma,
                                tail_area_level=tail_area_level, tail_window=tail_window,
                                psf_fwhm=psf_fwhm, nominal_cd=nominal_cd, dark_level=sign * float(dark_level),
                                flux_ratio_scale=flux_ratio_scale)


def _measure_peaks(img, signal, sign, *, peak_min_distance, **kw):
    """seeds="peaks" (subpx/cd.py:502-511): square boxes of 2 ceil(0.6 pitch) + 1 around each peak,
    no component ids, every hole reported by its fitted reach, no excluded features, and the
    deblend's own tile rule."""
    peaks, pitch = odb.detect_peaks(signal, min_distance=peak_min_distance)
    half = int(np.ceil(0.6 * pitch))
    rows = np.array([[cx - half, cy - half, 2 * half + 1, 2 * half + 1, cx, cy] for cx, cy in peaks],
                    dtype=np.float64).reshape(-1, 6)
    n = len(rows)
    return _deblend_and_measure(img, signal, sign, rows, np.full(n, -1, np.int32), np.ones(n, bool),
                                np.ones(n, bool), pitch, None, None, None, **kw)


def _deblend_and_measure(img, signal, sign, rows, ids, interior, by_reach, pitch, tile_px, exclude_mask, oversized, *,
                         methods, pad, n_angles, radial_step, fit_fraction, deblend_iterations, deblend_tolerance,
                         background_level, smooth_sigma, tail_area_level=0.2, tail_window=1.2, psf_fwhm=None,
                         nominal_cd=None, dark_level=0.0, flux_ratio_scale=None):
    """The deblend passes with seed revision and the measurements (subpx/cd.py:581-760)."""
    h, w = img.shape

    def build(rows_):
        seeds_ = rows_[:, 4:6].copy()
        lab_ = ov.voronoi_labels(seeds_, img.shape)
        masks_, origins_ = cell_stack(lab_, rows_, pad, img.shape)
        return seeds_, lab_, masks_, origins_

    seeds, cell_labels, masks, origins = build(rows)
    tiled = seeds
    level = None if background_level is None else sign * float(background_level)
    passes, added, dropped = [], 0, 0
    state = None
    for revision in range(3):
        exclude = exclude_mask
        final = revision == 2 or not np.isfinite(pitch)
        tile = tile_px if (seeds is tiled and tile_px is not None) else None
        state = odb.deblend(signal, seeds, masks, origins, iterations=deblend_iterations if final else
                            min(10, deblend_iterations), tile=tile, exclude=exclude, background_level=level,
                            tolerance=deblend_tolerance)
        passes.append(int(state.iterations))
        if final:
            break
        drop, new = odb.revise_seeds(signal, state, seeds, pitch, exclude=oversized)
        if not drop.any() and not len(new):
            if state.converged or state.iterations >= deblend_iterations:
                break
            state = odb.deblend(signal, seeds, masks, origins, iterations=deblend_iterations - state.iterations,
                                init=state.params, tile=tile, exclude=exclude, background_level=level,
                                tolerance=deblend_tolerance)
            passes.append(int(state.iterations))
            break
        half = int(np.ceil(0.6 * pitch))
        keep_s = ~drop
        rows = np.concatenate((rows[keep_s], np.array([[px - half, py - half, 2 * half + 1, 2 * half + 1, px, py]
                                                       for px, py in new], dtype=np.float64).reshape(-1, 6)))
        ids = np.concatenate((ids[keep_s], np.full(len(new), -1, np.int32)))
        interior = np.concatenate((interior[keep_s], np.ones(len(new), bool)))
        by_reach = np.concatenate((by_reach[keep_s], np.ones(len(new), bool)))
        added, dropped = added + len(new), dropped + int(drop.sum())
        seeds, cell_labels, masks, origins = build(rows)
    if by_reach.any():
        p = state.params[by_reach]
        c = p[:, 1:3] + origins[by_reach]
        reach = np.where(np.isfinite(p).all(axis=1), 2 * K * odb.sigma_major(p), np.inf)
        interior[by_reach] = (c[:, 0] - reach > 0) & (c[:, 0] + reach < w - 1) & (c[:, 1] - reach > 0) & \
            (c[:, 1] + reach < h - 1)
    report = np.flatnonzero(interior)
    cleaned = state.cleaned[report]
    from .invariant import HALF_AREA, TAIL_AREA

    measured = [m for m in methods if m not in ("gaussian", "projection", "disk", "flux_ratio")
                and m not in HALF_AREA and m not in TAIL_AREA]
    out = measure_cells(cleaned, masks[report], origins[report], seeds[report], methods=measured, n_angles=n_angles,
                        radial_step=radial_step, fit_fraction=fit_fraction, smooth_sigma=smooth_sigma) if measured else {}
    if "gaussian" in methods:
        out["gaussian"] = gaussian_method(state.params[report], state.status[report], cleaned, masks[report],
                                          origins[report], n_angles)
    if "projection" in methods:
        from .invariant import projection

        out["projection"] = projection(cleaned, masks[report], origins[report], n_angles)
    half = [m for m in methods if m in HALF_AREA]
    if half:
        from .invariant import half_areas

        out.update(half_areas(cleaned, masks[report], origins[report], n_angles, half))
    tails = [m for m in methods if m in TAIL_AREA]
    tail_info = {}
    if tails:
        from .invariant import tail_areas

        found = tail_areas(signal, state, masks, origins, report, n_angles, tails, level=tail_area_level,
                           window=tail_window, pitch=float(pitch) if np.isfinite(pitch) else None)
        tail_info = found.pop("_info")
        out.update(found)
    disks = [m for m in methods if m in ("disk", "flux_ratio")]
    if disks:
        from .disk import disk_methods

        found = disk_methods(signal, state, masks, origins, report, n_angles, disks, psf_fwhm_px=psf_fwhm,
                             nominal_cd_px=nominal_cd, dark_level=dark_level, flux_ratio_scale=flux_ratio_scale)
        tail_info.update(found.pop("_info"))
        out.update(found)
    out = {m: out[m] for m in methods}
    from scipy.ndimage import map_coordinates

    local = sign * map_coordinates(state.background_map, seeds[report].T[::-1], order=1, mode="nearest") \
        if len(report) else np.zeros(0)
    for r in out.values():
        r["metrics"]["background"][:] = local
    params_global = state.params.copy()
    params_global[:, 1:3] += origins
    remap = np.full(len(rows) + 1, -1, dtype=np.int32)
    remap[report] = np.arange(len(report), dtype=np.int32)
    return {"seeds": seeds[report], "cell_labels": remap[cell_labels], "measurements": out, "params": params_global,
            "report": report, "passes": passes, "iterations_used": sum(passes), "added": added, "dropped": dropped,
            "source": state.background_info.get("source"), "background_map": sign * state.background_map,
            "status": state.status[report], "pitch": pitch, "tail_info": tail_info}


def threshold_cells(img, *, threshold="otsu", invert=False, area_min=3, area_max=50, pad=3):
    """Seeds, cell masks and origins of thresholded components (subpx/cd.py:472-538: segmentation,
    area filter, Voronoi cells of the centroids, boxes grown by pad)."""
    img = np.asarray(img)
    t = osg.otsu_threshold(img) if threshold == "otsu" else osg.triangle_threshold(img)
    num, labels, stats, cents = osg.label_components(osg.binarize(img, t, invert), 8)
    area = stats[1:num, 4]
    keep = (area >= area_min) & (area <= area_max)
    rows = np.column_stack((stats[1:num, :4], cents[1:num])).astype(np.float64)[keep]
    seeds = rows[:, 4:6].copy()
    masks, origins = cell_stack(ov.voronoi_labels(seeds, img.shape), rows, pad, img.shape)
    return seeds, masks, origins
