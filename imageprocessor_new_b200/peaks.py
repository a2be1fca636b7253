"""Peak seeds on the device for arrays too dense to threshold (measure_cds(seeds="peaks")).

Follows estimate_pitch and detect_peaks (subpx/_cpu/deblend.py:570-630), reached from
subpx/cd.py:502-511 (which runs them on the host even for the reference's GPU backend). Every
per-pixel step runs in libsubpx_b200: the centred crop, the radial bins of its autocorrelation and
the pick of the first ring (spx_pitch_*), the separable Gaussian / maximum / minimum filters, the
row-major candidate compaction and the kept seeds' parabola refinement (spx_peak_*). The two
transforms of the autocorrelation are cuFFT's, through torch.fft on the current stream.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _device as dev
from . import _lib


def gaussian_weights(sigma: float) -> tuple[np.ndarray, int]:
    """scipy.ndimage's 1-D Gaussian kernel (truncate 4): radius int(4 sigma + 0.5) and
    exp(-0.5 / sigma^2 x^2) normalised to sum 1 (scipy.ndimage._filters._gaussian_kernel1d)."""
    radius = int(4.0 * float(sigma) + 0.5)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return phi / phi.sum(), radius


def estimate_pitch(img_d: torch.Tensor, sign: float, *, max_size: int = 1024) -> float:
    """Lattice pitch of the image (times sign) from the first ring of the radially averaged
    autocorrelation of its centred crop (subpx/_cpu/deblend.py:570-590)."""
    h, w = (int(v) for v in img_d.shape)
    ch, cw = min(h, max_size), min(w, max_size)
    stream = dev.stream_ptr()
    ws = dev.workspace(_lib.size("spx_pitch_workspace_bytes", h, w, max_size))
    padded = dev.empty((2 * ch, 2 * cw), torch.float64)
    _lib.call("spx_pitch_crop", img_d.data_ptr(), dev.dtype_code(img_d), float(sign), h, w, int(max_size),
              padded.data_ptr(), ws.data_ptr(), ws.numel(), stream)
    spectrum = torch.fft.rfft2(padded)
    power = spectrum.real.square() + spectrum.imag.square()
    autoc = torch.fft.irfft2(power, s=padded.shape).contiguous()
    pitch_d = dev.empty((1,), torch.float64)
    _lib.call("spx_pitch_from_autocorrelation", autoc.data_ptr(), 2 * ch, 2 * cw, min(ch, cw) // 2,
              pitch_d.data_ptr(), ws.data_ptr(), ws.numel(), stream)
    pitch = float(pitch_d.item())
    if not np.isfinite(pitch):
        raise ValueError("could not estimate the hole pitch; pass peak_min_distance explicitly")
    return pitch


def detect_peaks(img_d: torch.Tensor, sign: float, *, min_distance: float | None = None,
                 smooth_sigma: float | None = None, threshold: float = 0.25) -> tuple[np.ndarray, float]:
    """Local-maximum seeds [x, y] of sign * image and the pitch (subpx/_cpu/deblend.py:593-630):
    maxima of the smoothed signal over (2 floor(min_distance) + 1)^2 windows with positive
    prominence over the (2 ceil(pitch) + 1)^2 minimum, kept at >= threshold x the 90th percentile
    prominence, in row-major order, refined by the parabola through their neighbours."""
    h, w = (int(v) for v in img_d.shape)
    pitch = 2.0 * float(min_distance) if min_distance is not None else estimate_pitch(img_d, sign)
    if min_distance is None:
        min_distance = 0.5 * pitch
    if smooth_sigma is None:
        smooth_sigma = max(0.5, 0.1 * pitch)
    stream = dev.stream_ptr()
    signal = dev.empty((h, w), torch.float64)
    _lib.call("spx_signal_image", img_d.data_ptr(), dev.dtype_code(img_d), float(sign), h, w, signal.data_ptr(),
              stream)
    weights, radius = gaussian_weights(smooth_sigma)
    weights_d = dev.upload(weights)
    tmp = dev.empty((h, w), torch.float64)
    smooth = dev.empty((h, w), torch.float64)
    _lib.call("spx_gaussian_filter", signal.data_ptr(), h, w, weights_d.data_ptr(), radius, tmp.data_ptr(),
              smooth.data_ptr(), stream)
    maxf = signal  # the signal is no longer needed
    _lib.call("spx_maximum_filter", smooth.data_ptr(), h, w, max(1, int(np.floor(min_distance))), tmp.data_ptr(),
              maxf.data_ptr(), stream)
    minf = dev.empty((h, w), torch.float64)
    _lib.call("spx_minimum_filter", smooth.data_ptr(), h, w, int(np.ceil(pitch)), tmp.data_ptr(), minf.data_ptr(),
              stream)
    ws = dev.workspace(_lib.size("spx_peak_workspace_bytes", h, w))
    count = dev.empty((1,), torch.int32)
    cap = max(1024, (h * w) // max(1, (2 * max(1, int(np.floor(min_distance))) + 1) ** 2) * 2)
    while True:
        yx = dev.empty((cap, 2), torch.int32)
        prom = dev.empty((cap,), torch.float64)
        _lib.call("spx_peak_candidates", smooth.data_ptr(), maxf.data_ptr(), minf.data_ptr(), h, w, yx.data_ptr(),
                  prom.data_ptr(), cap, count.data_ptr(), ws.data_ptr(), ws.numel(), stream)
        n = dev.read_int(count)
        if n <= cap:
            break
        cap = n
    if n == 0:
        return np.zeros((0, 2)), pitch
    # np.percentile(prominence, 90) on the device ('linear'), then the kept seeds in order.
    from .deblend import quantile_device

    level = quantile_device(_lib.QuantileReq(prom.data_ptr(), 1, None, 0, n, 1, 0.9))
    out = dev.empty((n, 2), torch.float64)
    ws2 = dev.workspace(_lib.size("spx_peak_select_workspace_bytes", n))
    _lib.call("spx_peak_select", yx.data_ptr(), prom.data_ptr(), n, level.data_ptr(), float(threshold),
              smooth.data_ptr(), h, w, out.data_ptr(), count.data_ptr(), ws2.data_ptr(), ws2.numel(), stream)
    k = dev.read_int(count)
    return out[:k].cpu().numpy(), pitch
