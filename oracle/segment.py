"""Oracle: Otsu / triangle thresholds, binarisation, connected components (CPU, test infrastructure).

Reference call sites: subpx/_cpu/centers.py:247-266 (_segment_binary: cv2.threshold with
THRESH_OTSU / THRESH_TRIANGLE), subpx/_gpu/centers.py:1789-1796 (Otsu of img[::ds, ::ds] x thr_scale,
then a fixed threshold), subpx/_cpu/components.py:18-32 (cv2.connectedComponentsWithStats).
"""

from __future__ import annotations

import numpy as np

FLT_EPSILON = float(np.float32(np.finfo(np.float32).eps))


def histogram(img: np.ndarray) -> np.ndarray:
    nbins = 256 if img.dtype == np.uint8 else 65536
    return np.bincount(np.asarray(img).ravel(), minlength=nbins).astype(np.int64)


def otsu_threshold(img: np.ndarray) -> float:
    """OpenCV's Otsu threshold (getThreshVal_Otsu) of a uint8/uint16 image, as a whole number.

    For each bin i, with q1 = P(v <= i) and class means mu1, mu2, maximise q1 q2 (mu1 - mu2)^2; the
    first maximum wins; bins where min(q1, q2) < FLT_EPSILON or max(q1, q2) > 1 - FLT_EPSILON are
    skipped. The recurrences are evaluated in OpenCV's order so that the chosen bin is identical.
    """
    img = np.asarray(img)
    if img.dtype not in (np.uint8, np.uint16):
        raise ValueError("Otsu needs uint8 or uint16")
    return otsu_from_histogram(histogram(img), img.size)


def otsu_from_histogram(h: np.ndarray, total: int) -> float:
    """The Otsu scan of otsu_threshold on a histogram of `total` pixels (a sum of histograms of row
    shards gives the whole image's threshold)."""
    h = np.asarray(h, dtype=np.int64)
    scale = 1.0 / total
    mu = float(np.dot(np.arange(len(h), dtype=np.int64), h)) * scale  # exact integer sum
    nz = np.flatnonzero(h)
    if len(nz) == 0:
        return 0.0
    mu1 = q1 = 0.0
    max_sigma = max_val = 0.0
    hf = h.astype(np.float64)
    for i in range(int(nz[0]), int(nz[-1]) + 1):
        p_i = hf[i] * scale
        mu1 *= q1
        q1 += p_i
        q2 = 1.0 - q1
        if min(q1, q2) < FLT_EPSILON or max(q1, q2) > 1.0 - FLT_EPSILON:
            continue
        mu1 = (mu1 + i * p_i) / q1
        mu2 = (mu - q1 * mu1) / q2
        sigma = q1 * q2 * (mu1 - mu2) * (mu1 - mu2)
        if sigma > max_sigma:
            max_sigma, max_val = sigma, float(i)
    return max_val


def triangle_threshold(img: np.ndarray) -> float:
    """OpenCV's triangle threshold (getThreshVal_Triangle_8u) of a uint8 image."""
    img = np.asarray(img)
    if img.dtype != np.uint8:
        raise ValueError("triangle needs uint8")
    h = histogram(img).copy()
    n = 256
    nz = np.flatnonzero(h)
    left = int(nz[0]) if len(nz) else 0
    left = left - 1 if left > 0 else left
    right = 0
    for i in range(n - 1, 0, -1):
        if h[i] > 0:
            right = i
            break
    right = right + 1 if right < n - 1 else right
    max_ind = int(np.argmax(h))
    peak = int(h[max_ind])
    flipped = False
    if max_ind - left < right - max_ind:
        flipped = True
        h = h[::-1].copy()
        left = n - 1 - right
        max_ind = n - 1 - max_ind
    thresh, dist = float(left), 0.0
    a, b = float(peak), float(left - max_ind)
    for i in range(left + 1, max_ind + 1):
        d = a * i + b * float(h[i])
        if d > dist:
            dist, thresh = d, float(i)
    thresh -= 1
    if flipped:
        thresh = n - 1 - thresh
    return thresh


def binarize(img: np.ndarray, t: float, invert: bool = False) -> np.ndarray:
    """cv2.threshold(img, t, 255, THRESH_BINARY[_INV]) as a boolean foreground mask: img > t (<= t)."""
    v = np.asarray(img)
    return (v <= t) if invert else (v > t)


def morphology(fg: np.ndarray, morph_open: int = 0, morph_close: int = 0) -> np.ndarray:
    """cv2.morphologyEx(bw, MORPH_OPEN, k, iterations=morph_open) then MORPH_CLOSE with
    k = getStructuringElement(MORPH_ELLIPSE, (3, 3)) -- the 3x3 cross -- on a boolean mask
    (subpx/_cpu/centers.py:260-265). OPEN is `n` erosions then `n` dilations, CLOSE the reverse;
    pixels outside the image never change a minimum or a maximum (OpenCV's default border)."""
    m = np.asarray(fg, dtype=bool).copy()

    def erode(a):
        out = a.copy()
        out[1:, :] &= a[:-1, :]
        out[:-1, :] &= a[1:, :]
        out[:, 1:] &= a[:, :-1]
        out[:, :-1] &= a[:, 1:]
        return out

    def dilate(a):
        out = a.copy()
        out[1:, :] |= a[:-1, :]
        out[:-1, :] |= a[1:, :]
        out[:, 1:] |= a[:, :-1]
        out[:, :-1] |= a[:, 1:]
        return out

    for op, times in ((erode, morph_open), (dilate, morph_open), (dilate, morph_close), (erode, morph_close)):
        for _ in range(int(times)):
            m = op(m)
    return m


def label_components(fg: np.ndarray, connectivity: int = 8):
    """(num_labels, labels int32, stats (K+1, 5) int32, centroids (K+1, 2) f64) numbered as OpenCV:
    components ordered by their first 2x2 block in row-pair scan order (8-connectivity) or their
    first pixel in raster order (4-connectivity); label 0 is the background."""
    from scipy import ndimage

    fg = np.asarray(fg, dtype=bool)
    h, w = fg.shape
    structure = np.ones((3, 3), int) if connectivity == 8 else None
    lab, n = ndimage.label(fg, structure=structure)
    yy, xx = np.indices(fg.shape)
    if connectivity == 8:
        key = (yy // 2).astype(np.int64) * ((w + 1) // 2) + (xx // 2)
    else:
        key = yy.astype(np.int64) * w + xx
    first = np.full(n + 1, np.iinfo(np.int64).max)
    np.minimum.at(first, lab.ravel(), key.ravel())
    order = np.argsort(first[1:], kind="stable")
    remap = np.zeros(n + 1, np.int64)
    remap[1 + order] = np.arange(1, n + 1)
    labels = remap[lab].astype(np.int32)
    flat = labels.ravel()
    area = np.bincount(flat, minlength=n + 1)
    sx = np.bincount(flat, weights=xx.ravel().astype(np.float64), minlength=n + 1)
    sy = np.bincount(flat, weights=yy.ravel().astype(np.float64), minlength=n + 1)
    xmin = np.full(n + 1, w, np.int64)
    ymin = np.full(n + 1, h, np.int64)
    xmax = np.full(n + 1, -1, np.int64)
    ymax = np.full(n + 1, -1, np.int64)
    np.minimum.at(xmin, flat, xx.ravel())
    np.minimum.at(ymin, flat, yy.ravel())
    np.maximum.at(xmax, flat, xx.ravel())
    np.maximum.at(ymax, flat, yy.ravel())
    stats = np.column_stack((xmin, ymin, xmax - xmin + 1, ymax - ymin + 1, area)).astype(np.int32)
    with np.errstate(invalid="ignore", divide="ignore"):
        centroids = np.column_stack((sx / area, sy / area))
    empty = area == 0
    stats[empty, :4] = 0
    return n + 1, labels, stats, centroids
