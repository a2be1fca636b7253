"""The FP32 LM arithmetic (FP32 per-pixel sums, FP64 solve and acceptance, stop at a 1e-7 relative
cost drop) against the FP64 one, which follows the reference: same statuses, centres within 1e-3 px,
Gaussian sigmas and Gaussian-FWHM CDs within 2e-3 px."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [4, 9])
def test_fp32_initial_fits_match_fp64(seed):
    from imageprocessor_new_b200 import warmstart as ws

    page, _ = ws.synth_page(seed, 1536)
    cells = ws.page_cells(page)
    assert cells.n > 500
    p64, s64, i64, _, _ = (a.cpu().numpy() for a in ws.initial_fits(page, cells))
    p32, s32, i32, _, _ = (a.cpu().numpy() for a in ws.initial_fits(page, cells, precision="fp32"))
    assert (s32 == s64).mean() >= 0.999
    ok = (s32 == 0) & (s64 == 0)
    assert ok.sum() > 0.9 * cells.n
    assert np.abs(p32[ok, 1:3] - p64[ok, 1:3]).max() <= 1e-3
    # sigma along each axis of the precision factor
    assert np.abs(np.exp(-p32[ok, 3]) - np.exp(-p64[ok, 3])).max() <= 2e-3
    assert np.abs(np.exp(-p32[ok, 5]) - np.exp(-p64[ok, 5])).max() <= 2e-3
    # The FP32 rule stops earlier on these large-residual fits.
    assert i32.mean() < i64.mean()


def test_fp64_fits_are_deterministic():
    """Two FP64 runs over the device work queue give the same bits (cells are fitted in whatever order
    the warps take them; each cell's arithmetic does not depend on it)."""
    from imageprocessor_new_b200 import warmstart as ws

    page, _ = ws.synth_page(4, 1024)
    cells = ws.page_cells(page)
    a = [t.cpu().numpy() for t in ws.initial_fits(page, cells)]
    b = [t.cpu().numpy() for t in ws.initial_fits(page, cells, precision="fp64")]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_fp32_measure_cds_gaussian_matches_fp64():
    import torch

    from imageprocessor_new_b200 import measure_cds, synthetic

    page = synthetic.page_staggered(0, shape=(1024, 1024)).image
    page_d = torch.from_numpy(page).cuda()
    kw = dict(methods=("gaussian",), area_max=400, backend="gpu")
    r64 = measure_cds(page_d, **kw)
    r32 = measure_cds(page_d, fit_precision="fp32", **kw)
    assert r32.meta["fit_precision"] == "fp32"
    assert np.array_equal(r64.seeds_xy, r32.seeds_xy)
    a, b = r32.measurements["gaussian"], r64.measurements["gaussian"]
    assert np.array_equal(a.valid, b.valid)
    v = a.valid
    assert v.sum() > 1000
    assert np.abs(a.centers_xy[v] - b.centers_xy[v]).max() <= 1e-3
    for m in ("cd_equivalent_px", "fwhm_major_px", "fwhm_minor_px"):
        assert np.abs(a.metrics[m][v] - b.metrics[m][v]).max() <= 2e-3, m
