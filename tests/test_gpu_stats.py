"""Device order statistics and background sampling used by the deblending loop.

spx_quantiles replaces np.median / np.percentile(q, method="linear") of subpx/_cpu/deblend.py:463-464
and :517; spx_background_at replaces map_coordinates(map, [y, x], order=1, mode="nearest") of
subpx/cd.py:719-721. Both are checked bit-exact against numpy / scipy on the same inputs.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(reqs_spec):
    import torch

    from imageprocessor_new_b200 import _lib
    from imageprocessor_new_b200.deblend import quantiles

    keep, reqs = [], []
    for values, stride, mask, finite_only, mode, q in reqs_spec:
        v = torch.from_numpy(np.ascontiguousarray(values)).cuda()
        m = None if mask is None else torch.from_numpy(mask.astype(np.uint8)).cuda()
        keep += [v, m]
        n = v.numel() // stride
        reqs.append(_lib.QuantileReq(v.data_ptr(), stride, None if m is None else m.data_ptr(), finite_only, n, mode, q))
    out = quantiles(reqs)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 10, 1001, 4096, 116_793])
def test_median_and_percentile_match_numpy(n):
    rng = np.random.default_rng(n)
    vals = rng.normal(3.0, 2.0, n)
    vals[rng.random(n) < 0.1] = 1.25          # ties
    mask = rng.random(n) < 0.7
    steps = np.abs(rng.normal(0, 1e-3, n))
    steps[rng.random(n) < 0.05] = np.nan      # failed fits
    steps[rng.random(n) < 0.01] = np.inf
    params = rng.normal(0, 1, (n, 6))
    out = _run([(vals, 1, None, 0, 0, 0.0), (vals, 1, mask, 0, 0, 0.0), (steps, 1, None, 1, 1, 99 / 100),
                (params, 6, mask, 0, 0, 0.0), (vals, 1, None, 0, 1, 0.5)])
    assert out[0, 0] == np.median(vals) and out[0, 1] == n
    if mask.any():
        assert out[1, 0] == np.median(vals[mask]) and out[1, 1] == mask.sum()
        assert out[3, 0] == np.median(params[mask, 0])
    else:
        assert np.isnan(out[1, 0]) and out[1, 1] == 0
    ok = np.isfinite(steps)
    if ok.any():
        assert out[2, 0] == np.percentile(steps[ok], 99) and out[2, 1] == ok.sum()
    assert out[4, 0] == np.percentile(vals, 50)


def test_median_with_nan_is_nan_and_empty_selection():
    vals = np.array([1.0, np.nan, 3.0, -0.0, 0.0])
    out = _run([(vals, 1, None, 0, 0, 0.0), (vals, 1, np.zeros(5, bool), 0, 0, 0.0),
                (vals, 1, None, 1, 0, 0.0)])
    assert np.isnan(out[0, 0]) and np.isnan(np.median(vals))
    assert np.isnan(out[1, 0]) and out[1, 1] == 0
    assert out[2, 0] == np.median(vals[np.isfinite(vals)])


def test_background_at_matches_map_coordinates():
    import torch
    from scipy import ndimage

    from imageprocessor_new_b200 import deblend

    shape = (300, 410)
    bg = deblend.Background(shape, 64)
    rng = np.random.default_rng(3)
    bg.set_medians(rng.normal(1000.0, 25.0, (bg.ny, bg.nx)))
    full = bg.host_map()
    pts = np.column_stack([rng.uniform(-3, shape[1] + 3, 5000), rng.uniform(-3, shape[0] + 3, 5000)])
    pts[:10] = np.round(pts[:10])             # integer positions
    got = bg.at_points(torch.from_numpy(pts).cuda(), -1.0)
    want = -ndimage.map_coordinates(full, [pts[:, 1], pts[:, 0]], order=1, mode="nearest")
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)
    fixed = deblend.Background(shape, 64).set_fixed(12.5)
    want = ndimage.map_coordinates(np.full(shape, 12.5), [pts[:, 1], pts[:, 0]], order=1, mode="nearest")
    np.testing.assert_allclose(fixed.at_points(torch.from_numpy(pts).cuda()), want, rtol=0, atol=1e-9)
