"""The benchmark configurations' own pipelines on the GPU against the oracle, at full size or on a
large crop: the config-1 contact-hole page through measure_cds, a 1024 x 1024 staggered page of the
config-2 kind through all three CD methods, and tiled detection with the config-3 band geometry
(tile_h 8192, overlap 128) across two band seams.

Tolerances: cells, seeds, labels and statuses exact; centres within 1e-3 px and CDs within
2e-3 px of the oracle (FP64 sums in another order, FP32 ray samples).
"""

import numpy as np
import pytest

from oracle import cd as ocd
from oracle import centers as oc

pytestmark = pytest.mark.gpu


def _compare_cds(res, ref, methods):
    np.testing.assert_array_equal(res.seeds_xy, ref["seeds"])
    np.testing.assert_array_equal(res.cell_labels, ref["cell_labels"])
    assert res.meta["deblend_pass_iterations"] == ref["passes"]
    # FP64 sums in another order: positions and log-widths within 1e-6, amplitudes (thousands of
    # counts) within 1e-7 relative (a fit ends where the 1e-12 cost rule stops it).
    got_p, want_p = res.deblend_model["params"], ref["params"]
    np.testing.assert_allclose(got_p[:, 1:], want_p[:, 1:], rtol=0, atol=1e-6)
    np.testing.assert_allclose(got_p[:, 0], want_p[:, 0], rtol=1e-7, atol=1e-6)
    for m in methods:
        got, want = res.measurements[m], ref["measurements"][m]
        np.testing.assert_array_equal(got.status, want["status"], err_msg=m)
        a, b = got.metrics["cd_equivalent_px"], want["metrics"]["cd_equivalent_px"]
        assert np.array_equal(np.isnan(a), np.isnan(b)), m
        ok = ~np.isnan(a)
        assert ok.sum() >= 0.9 * len(a), m
        assert np.abs(a[ok] - b[ok]).max() <= 2e-3, (m, np.abs(a[ok] - b[ok]).max())
        fin = np.isfinite(want["centers"]).all(axis=1)
        assert np.array_equal(fin, np.isfinite(got.centers_xy).all(axis=1)), m
        assert np.abs(got.centers_xy[fin] - want["centers"][fin]).max() <= 1e-3, m


def test_config1_page_measure_cds_matches_oracle():
    """Config 1: the 1024 x 1024 uint16 contact-hole page (32 x 32 holes, pitch 32, d 14),
    detect_centers(refine="logquad") and measure_cds with the Gaussian-FWHM methods."""
    from imageprocessor_new_b200 import detect_centers, measure_cds, synthetic

    page = synthetic.page_square(0).image
    got = detect_centers(page, backend="gpu", threshold="otsu", refine="logquad", area_max=400).centers_xy
    want = oc.detect_centers(page, threshold="otsu", refine_method="logquad", area_max=400)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)
    methods = ("gaussian", "logquad")
    res = measure_cds(page, backend="gpu", methods=methods, threshold="otsu", area_max=400)
    ref = ocd.measure_cds(page, methods=methods, threshold="otsu", area_max=400)
    assert len(ref["seeds"]) >= 900
    _compare_cds(res, ref, methods)


def test_config2_staggered_page_all_cd_methods_match_oracle():
    """Config 2's page kind (staggered, pitch 24, d 12 +- 5 %, sigma 1.2, N(0, 100) read noise,
    border-clipped cells kept) at 1024 x 1024: the three refiners and the three CD methods."""
    from imageprocessor_new_b200 import detect_centers, measure_cds, synthetic

    page = synthetic.page_staggered(0, shape=(1024, 1024)).image
    for refine in ("weighted", "logquad", "edge_gradmoment"):
        got = detect_centers(page, backend="gpu", threshold="otsu", refine=refine, area_max=400).centers_xy
        want = oc.detect_centers(page, threshold="otsu", refine_method=refine, area_max=400)
        assert got.shape == want.shape, refine
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9, err_msg=refine)
    methods = ("gaussian", "gradient", "halfmax")
    res = measure_cds(page, backend="gpu", methods=methods, area_max=400)
    ref = ocd.measure_cds(page, methods=methods, area_max=400)
    assert len(ref["seeds"]) >= 1500
    _compare_cds(res, ref, methods)


def test_config3_band_seams_match_oracle_tiled_rules():
    """Config 3's band geometry on a 16512 x 512 strip (pitch 20, d 10 +- 4 %, sigma 1.0, +-15 %
    illumination): bands [0, 8192), [8064, 16256), [16128, 16512) with the keep rule at both seams,
    the global Otsu of img[::4, ::4] x 0.8 and the dedupe, against the oracle's tiled rules."""
    from imageprocessor_new_b200 import detect_centers, synthetic

    rng = np.random.default_rng(3)
    shape = (16512, 512)
    centers = synthetic.square_grid(shape, 20.0, rng)
    d = 10.0 * (1.0 + rng.uniform(-0.04, 0.04, len(centers)))
    yy, xx = np.indices(shape, dtype=np.float64)
    gain = 1.0 + 0.15 * np.sin(2 * np.pi * xx / 8192) * np.sin(2 * np.pi * yy / 8192)
    clean = synthetic.render(shape, centers, d, 1.0, amplitude=3000.0, background=1000.0, gain=gain)
    page = synthetic.add_noise(clean, rng, read_noise=20.0)
    kw = dict(threshold="otsu", area_max=400)
    res = detect_centers(page, backend="gpu", tile_h=8192, overlap=128, threshold_mode="global", refine="auto", **kw)
    want = oc.detect_tiled(page, tile_h=8192, overlap=128, threshold_mode="global", refine_method="auto", **kw)
    assert len(want) >= 0.98 * len(centers)
    key = lambda a: a[np.lexsort((a[:, 1], a[:, 0]))]
    got = res.centers_xy
    assert got.shape == want.shape
    np.testing.assert_allclose(key(got), key(want), rtol=0, atol=1e-9)
    # Holes on both seams (the keep rule's band limits 8128 and 16192) are found once each.
    for seam in (8192 - 64, 16256 - 64):
        near_want = np.abs(want[:, 1] - seam) < 40
        near_got = np.abs(got[:, 1] - seam) < 40
        assert near_want.sum() > 0 and near_got.sum() == near_want.sum()
