"""Peak seeding on the device (seeds="peaks") against the oracle's restatement of estimate_pitch and
detect_peaks (subpx/_cpu/deblend.py:570-630): the pitch of the autocorrelation ring to 1e-9
relative (cuFFT against pocketfft), the same seeds in the same (row-major) order to 1e-9 px, and
the minimum filter of the prominence bit-exact against SciPy."""

import numpy as np
import pytest

from oracle import deblend as odb

pytestmark = pytest.mark.gpu


def _lattices():
    from imageprocessor_new_b200 import synthetic

    out = {f"lattice{r}": synthetic.gaussian_lattice(r, seed=4)[0] for r in (1.4, 1.6, 2.0, 2.67)}
    out["faint"] = synthetic.gaussian_lattice(2.0, faint=6, faint_amplitude=0.26, seed=3)[0]
    page = synthetic.page_square(1, shape=(300, 1100)).image  # crop wider than max_size in x
    out["page_u16"] = page
    return out


@pytest.mark.parametrize("name", list(_lattices()))
def test_pitch_and_peaks_match_oracle(name):
    import torch

    from imageprocessor_new_b200 import peaks

    img = _lattices()[name]
    img_d = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    signal = img.astype(np.float64)
    want_pitch = odb.estimate_pitch(signal)
    got_pitch = peaks.estimate_pitch(img_d, 1.0)
    assert got_pitch == pytest.approx(want_pitch, rel=1e-9)
    want, wp = odb.detect_peaks(signal)
    got, gp = peaks.detect_peaks(img_d, 1.0)
    assert gp == pytest.approx(wp, rel=1e-9)
    assert got.shape == want.shape and len(want) > 10
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)


def test_peaks_of_inverted_image_with_given_distance():
    import torch

    from imageprocessor_new_b200 import peaks, synthetic

    img = 100.0 - synthetic.gaussian_lattice(2.0, seed=2)[0]
    img_d = torch.from_numpy(img).cuda()
    want, wp = odb.detect_peaks(-img, min_distance=3.0)
    got, gp = peaks.detect_peaks(img_d, -1.0, min_distance=3.0)
    assert gp == wp == 6.0
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)


@pytest.mark.parametrize("shape,radius", [((300, 517), 6), ((64, 2100), 1), ((90, 120), 230)])
def test_minimum_filter_matches_scipy(shape, radius):
    import torch
    from scipy import ndimage

    from imageprocessor_new_b200 import _lib

    rng = np.random.default_rng(radius)
    img = rng.normal(0, 50, shape)
    d = torch.from_numpy(img).cuda()
    tmp, out = torch.empty_like(d), torch.empty_like(d)
    _lib.call("spx_minimum_filter", d.data_ptr(), shape[0], shape[1], radius, tmp.data_ptr(), out.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(out.cpu().numpy(), ndimage.minimum_filter(img, size=2 * radius + 1, mode="nearest"))


def test_pitch_failure_raises_value_error():
    import torch

    from imageprocessor_new_b200 import peaks

    flat = torch.full((64, 64), 7, dtype=torch.uint16, device="cuda")
    with pytest.raises(ValueError, match="pass peak_min_distance"):
        peaks.estimate_pitch(flat, 1.0)
