"""The seed-revision filters and the feature masks against SciPy / NumPy on the same inputs.

spx_gaussian_filter restates scipy.ndimage.gaussian_filter(mode="nearest") with the weights the
caller passes (subpx/_cpu/deblend.py:556) and spx_maximum_filter restates maximum_filter (:558);
spx_label_mask is the per-label flag lookup with cross dilations of subpx/cd.py:411-421, 489-491.
Both shared-memory tile paths (radius <= 200) and the direct path (larger radii) are covered.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _weights(sigma):
    radius = int(4.0 * sigma + 0.5)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return phi / phi.sum(), radius


@pytest.mark.parametrize("shape,sigma,size_r", [((300, 517), 2.4, 12), ((64, 2100), 0.5, 1), ((1030, 40), 6.0, 30),
                                                 ((90, 120), 55.0, 230)])
def test_gaussian_and_maximum_filters_match_scipy(shape, sigma, size_r):
    import torch
    from scipy import ndimage

    from imageprocessor_new_b200 import _lib

    rng = np.random.default_rng(int(sigma * 10))
    img = rng.normal(0, 50, shape)
    img[rng.random(shape) < 0.01] += 900.0
    w, radius = _weights(sigma)
    d = torch.from_numpy(img).cuda()
    wd = torch.from_numpy(w).cuda()
    tmp = torch.empty_like(d)
    out = torch.empty_like(d)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.call("spx_gaussian_filter", d.data_ptr(), shape[0], shape[1], wd.data_ptr(), radius, tmp.data_ptr(),
              out.data_ptr(), stream)
    want = ndimage.correlate1d(ndimage.correlate1d(img, w, axis=0, mode="nearest"), w, axis=1, mode="nearest")
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-14, atol=1e-11)
    _lib.call("spx_maximum_filter", d.data_ptr(), shape[0], shape[1], size_r, tmp.data_ptr(), out.data_ptr(),
              stream)
    want = ndimage.maximum_filter(img, size=2 * size_r + 1, mode="nearest")
    np.testing.assert_array_equal(out.cpu().numpy(), want)


@pytest.mark.parametrize("shape,dilations", [((200, 256), 2), ((77, 131), 2), ((64, 64), 0), ((33, 40), 3)])
def test_label_mask_dilations(shape, dilations):
    import torch
    from scipy import ndimage

    from imageprocessor_new_b200 import _lib

    rng = np.random.default_rng(dilations + shape[1])
    labels = rng.integers(0, 40, shape).astype(np.int32)
    labels[rng.random(shape) < 0.8] = 0
    flags = (rng.random(40) < 0.4).astype(np.uint8)
    flags[0] = 0
    want = flags[labels].astype(bool)
    cross = ndimage.generate_binary_structure(2, 1)
    for _ in range(dilations):
        want = ndimage.binary_dilation(want, structure=cross)
    ld = torch.from_numpy(labels).cuda()
    fd = torch.from_numpy(flags).cuda()
    out = torch.empty(shape, dtype=torch.uint8, device="cuda")
    tmp = torch.empty_like(out)
    _lib.call("spx_label_mask", ld.data_ptr(), fd.data_ptr(), shape[0], shape[1], dilations, out.data_ptr(),
              tmp.data_ptr(), torch.cuda.current_stream().cuda_stream)
    got = out.cpu().numpy()
    assert set(np.unique(got)) <= {0, 1}
    np.testing.assert_array_equal(got.astype(bool), want)
