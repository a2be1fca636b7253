"""Seeded synthetic contact-hole pages: blurred discs on a background, with Poisson and read noise.

Test and benchmark data only. Each hole is a uniform disc of diameter d blurred by an isotropic
Gaussian of sigma s; its light at distance r from the centre is the disc-Gaussian convolution

    I(r) = int_0^R (rho / s^2) exp(-(r^2 + rho^2) / (2 s^2)) I0(r rho / s^2) d rho,   R = d / 2,

tabulated once per (R, s) and sampled at pixel centres. The named workloads:

* ``page_square``   1024 x 1024 uint16, 32 x 32 square grid, pitch 32, d 14 + N(0, 0.7), sigma 1.5,
                    3000 counts on 1000, Poisson + N(0, 20) read noise.
* ``page_staggered`` 8192 x 8192 uint16 staggered array (pitch 24 x 24, odd rows shifted 12), d 12 +- 5 %, sigma 1.2,
                    3000 on 1000, N(0, 100) read noise (SNR ~30), ~116k holes incl. border-clipped.
* ``page_large_device`` 32768 x 32768 uint16 square array, pitch 20, d 10 +- 4 %, sigma 1.0, slow
                    +-15 % sinusoidal illumination of the hole contrast, ~2.7M holes, rendered on the
                    GPU (pixel coverage of each disc sampled 4 x 4, blurred, noise added on the device).
* ``gaussian_lattice`` the Gaussian-spot lattice of the reference's GPU tests (amplitude 50 on 20).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Page:
    image: np.ndarray
    centers: np.ndarray  # (N, 2) true [x, y]
    diameters: np.ndarray  # (N,)
    meta: dict


def _profile_table(radius: float, sigma: float, r_max: float, step: float = 0.02):
    from scipy.special import i0e

    r = np.arange(0.0, r_max + step, step)
    rho = np.linspace(0.0, radius, 401)
    # exp(-(r^2 + rho^2)/(2 s^2)) I0(r rho / s^2) = exp(-(r - rho)^2 / (2 s^2)) i0e(r rho / s^2)
    rr, pp = r[:, None], rho[None, :]
    integrand = (pp / sigma**2) * np.exp(-((rr - pp) ** 2) / (2 * sigma**2)) * i0e(rr * pp / sigma**2)
    values = np.trapezoid(integrand, rho, axis=1)
    return r, values


def render(shape, centers, diameters, sigma, *, amplitude=3000.0, background=1000.0, gain=None,
           chunk: int = 4096) -> np.ndarray:
    """Noise-free float64 page: background + amplitude * sum of blurred discs (x gain map if given)."""
    h, w = shape
    page = np.zeros(h * w, dtype=np.float64)
    centers = np.asarray(centers, dtype=np.float64).reshape(-1, 2)
    diameters = np.broadcast_to(np.asarray(diameters, dtype=np.float64), (len(centers),))
    if len(centers):
        reach = int(np.ceil(0.5 * diameters.max() + 5 * sigma)) + 1
        off = np.arange(-reach, reach + 1)
        # Tabulate on a grid of radii 0.05 px apart at most (the nearest one renders a hole).
        rad = 0.5 * diameters
        lo, hi = rad.min(), rad.max()
        buckets = np.linspace(lo, hi, int(np.ceil((hi - lo) / 0.05)) + 1) if hi > lo else np.array([lo])
        tables = [_profile_table(b, sigma, reach * 1.5) for b in buckets]
        table_r = tables[0][0]
        table_v = np.stack([t[1] for t in tables])
        step = table_r[1] - table_r[0]
        which = np.clip(np.rint((rad - lo) / max(hi - lo, 1e-12) * (len(buckets) - 1)).astype(int), 0,
                        len(buckets) - 1) if len(buckets) > 1 else np.zeros(len(rad), int)
        for start in range(0, len(centers), chunk):
            c = centers[start:start + chunk]
            k = which[start:start + chunk]
            ix = np.rint(c[:, 0]).astype(np.int64)[:, None, None] + off[None, None, :]
            iy = np.rint(c[:, 1]).astype(np.int64)[:, None, None] + off[None, :, None]
            ix, iy = np.broadcast_arrays(ix, iy)
            r = np.hypot(ix - c[:, 0, None, None], iy - c[:, 1, None, None])
            pos = r / step
            i0 = np.minimum(pos.astype(np.int64), len(table_r) - 2)
            t = pos - i0
            vals = (1 - t) * table_v[k[:, None, None], i0] + t * table_v[k[:, None, None], i0 + 1]
            ok = (ix >= 0) & (ix < w) & (iy >= 0) & (iy < h)
            page += np.bincount((iy * w + ix)[ok], weights=vals[ok], minlength=h * w)
    page = page.reshape(h, w) * amplitude
    if gain is not None:
        page *= gain
    return page + background


def add_noise(clean: np.ndarray, rng, *, read_noise: float, poisson: bool = True, bits: int = 16):
    noisy = rng.poisson(np.clip(clean, 0, None)).astype(np.float64) if poisson else clean.copy()
    if read_noise > 0:
        noisy += rng.normal(0.0, read_noise, clean.shape)
    top = 2**bits - 1
    return np.clip(np.rint(noisy), 0, top).astype(np.uint16 if bits > 8 else np.uint8)


def square_grid(shape, pitch, rng, *, jitter=0.5, margin=None):
    h, w = shape
    m = pitch / 2 if margin is None else margin
    xs = np.arange(m, w, pitch)
    ys = np.arange(m, h, pitch)
    gx, gy = np.meshgrid(xs, ys)
    c = np.column_stack((gx.ravel(), gy.ravel())).astype(np.float64)
    return c + rng.uniform(-jitter, jitter, c.shape)


def staggered_grid(shape, pitch, rng, *, pitch_y=None, jitter=0.5):
    """Rows ``pitch_y`` apart (default: pitch), odd rows shifted by half a pitch; holes cut by the
    border are kept."""
    h, w = shape
    dy = pitch if pitch_y is None else pitch_y
    rows = np.arange(0, h + dy, dy)
    pts = []
    for j, y in enumerate(rows):
        x0 = (pitch / 2) * (j % 2)
        xs = np.arange(x0, w + pitch, pitch)
        pts.append(np.column_stack((xs, np.full(len(xs), y))))
    c = np.concatenate(pts).astype(np.float64)
    c = c[(c[:, 0] < w + 2) & (c[:, 1] < h + 2)]
    return c + rng.uniform(-jitter, jitter, c.shape)


def page_square(seed: int = 0, shape=(1024, 1024)) -> Page:
    rng = np.random.default_rng(seed)
    centers = square_grid(shape, 32.0, rng)
    d = 14.0 + rng.normal(0.0, 0.7, len(centers))
    clean = render(shape, centers, d, 1.5, amplitude=3000.0, background=1000.0)
    img = add_noise(clean, rng, read_noise=20.0)
    return Page(img, centers, d, dict(name="page_square", pitch=32.0, sigma=1.5, seed=seed))


def page_staggered(seed: int = 0, shape=(8192, 8192)) -> Page:
    rng = np.random.default_rng(seed)
    centers = staggered_grid(shape, 24.0, rng)
    d = 12.0 * (1.0 + rng.uniform(-0.05, 0.05, len(centers)))
    clean = render(shape, centers, d, 1.2, amplitude=3000.0, background=1000.0)
    img = add_noise(clean, rng, read_noise=100.0, poisson=False)
    return Page(img, centers, d, dict(name="page_staggered", pitch=24.0, sigma=1.2, seed=seed))


def gaussian_lattice(ratio: float, *, snr: float = 20, shape=(120, 240), seed: int = 0, fwhm: float = 4.0,
                     missing: float = 0.0, small: int = 0, faint: int = 0, faint_amplitude: float = 0.28):
    """Staggered Gaussian spots (amplitude 50 on 20) with a 15 px margin, as the reference's tests
    build them (tests/test_cd_gpu.py:23-35, tests/test_deblend.py:15-33). ``missing`` drops that
    fraction of the spots at random; ``small`` interior spots get sigma 1.1 px (thresholding misses
    them, tests/test_deblend_variants.py:27-43) and ``faint`` others get ``faint_amplitude`` x the
    amplitude (peak seeding finds them, seed revision drops them). Returns (float64 image, centers)."""
    rng = np.random.default_rng(seed)
    pitch, sigma0 = ratio * fwhm, fwhm / (2 * np.sqrt(2 * np.log(2)))
    xx, yy = np.meshgrid(np.arange(15, shape[1] - 15, pitch), np.arange(15, shape[0] - 15, pitch))
    xx[1::2] += pitch / 2
    centers = np.column_stack((xx.ravel(), yy.ravel()))
    centers = centers[centers[:, 0] < shape[1] - 15]
    if missing:
        centers = centers[rng.random(len(centers)) >= missing]
    sigma = np.full(len(centers), sigma0)
    amp = np.full(len(centers), 50.0)
    if small or faint:
        inner = np.flatnonzero((np.abs(centers[:, 0] - shape[1] / 2) < shape[1] / 2 - 40)
                               & (np.abs(centers[:, 1] - shape[0] / 2) < shape[0] / 2 - 30))
        pick = rng.choice(inner, small + faint, replace=False)
        sigma[pick[:small]] = 1.1
        amp[pick[small:]] *= faint_amplitude
    y, x = np.indices(shape, dtype=float)
    image = np.full(shape, 20.0)
    for (cx, cy), s, a in zip(centers, sigma, amp):
        image += a * np.exp(-0.5 * ((x - cx) ** 2 + (y - cy) ** 2) / s**2)
    return image + (rng.normal(0, 50 / snr, shape) if snr else 0), centers


def dot_grid(rows=4, cols=4, spacing=20, dot_size=3, margin=10):
    """Bright square dots on black (uint8), with their exact centres."""
    h = 2 * margin + (rows - 1) * spacing + dot_size
    w = 2 * margin + (cols - 1) * spacing + dot_size
    img = np.zeros((h, w), dtype=np.uint8)
    expected = []
    for r in range(rows):
        for c in range(cols):
            y0, x0 = margin + r * spacing, margin + c * spacing
            img[y0:y0 + dot_size, x0:x0 + dot_size] = 255
            expected.append([x0 + (dot_size - 1) / 2.0, y0 + (dot_size - 1) / 2.0])
    return img, np.array(expected, dtype=np.float64)


def page_large_device(seed: int = 0, size: int = 32768, *, pitch: float = 20.0, d: float = 10.0, sigma: float = 1.0,
                      amplitude: float = 3000.0, background: float = 1000.0, read_noise: float = 20.0):
    """The tiled-detection page on the device (uint16 torch tensor) and its true centres (host)."""
    import ctypes

    import torch

    from . import _device as dev
    from . import _lib

    rng = np.random.default_rng(seed)
    centers = square_grid((size, size), pitch, rng)
    n = len(centers)
    di = d * (1.0 + rng.uniform(-0.04, 0.04, n))
    holes = np.column_stack((centers, di / 2, di / 2, np.zeros(n), np.full(n, 2.0)))
    cell = float(np.ceil(pitch))
    gw = int(np.ceil(size / cell)) + 1
    gx = np.clip(np.floor(holes[:, 0] / cell).astype(np.int64), 0, gw - 1)
    gy = np.clip(np.floor(holes[:, 1] / cell).astype(np.int64), 0, gw - 1)
    key = gy * gw + gx
    order = np.argsort(key, kind="stable")
    start = np.zeros(gw * gw + 1, np.int64)
    np.add.at(start, key + 1, 1)
    start = np.cumsum(start).astype(np.int32)
    holes_d = dev.upload(np.ascontiguousarray(holes))
    start_d, ids_d = dev.upload(start), dev.upload(order.astype(np.int32))
    s = dev.stream_ptr()
    cov = dev.empty((size, size), torch.float64)
    _lib.call("spx_hole_coverage", size, size, holes_d.data_ptr(), start_d.data_ptr(), ids_d.data_ptr(), gw, gw, cell,
              4, cov.data_ptr(), s)
    radius = int(4.0 * sigma + 0.5)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    wts = dev.upload(phi / phi.sum())
    tmp = dev.empty((size, size), torch.float64)
    _lib.call("spx_gaussian_filter", cov.data_ptr(), size, size, wts.data_ptr(), radius, tmp.data_ptr(),
              cov.data_ptr(), s)
    del tmp
    wave = torch.sin(2.0 * np.pi / 8192.0 * torch.arange(size, dtype=torch.float64, device="cuda"))
    for r0 in range(0, size, 1024):  # cov *= 1 + 0.15 sin(2 pi y / 8192) sin(2 pi x / 8192), in row blocks
        cov[r0:r0 + 1024] *= 1.0 + 0.15 * wave[r0:r0 + 1024, None] * wave[None, :]
    page = dev.empty((size, size), torch.uint16)
    _lib.call("spx_page_finish", cov.data_ptr(), size * size, float(background), float(amplitude), float(read_noise),
              ctypes.c_ulonglong(int(rng.integers(0, 2 ** 63))), page.data_ptr(), s)
    return page, centers
