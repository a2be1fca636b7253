"""measure_cds on the GPU against the reference's own CPU measure_cds (golden fixtures).

The fixtures (tests/golden/make_golden.py) cover threshold seeding on lattices, contact-hole pages
and an inverted page; peak seeding on a pitch / FWHM 1.4 array (lattice14) and on dark holes with a
fixed background level; seed revision that drops seeds (drop_peaks) and adds them (add_threshold),
each with two deblend passes; and smoothed radial profiles (page_smooth, smooth_sigma = 1).
"""

import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = ("lattice2", "lattice14", "page", "staggered", "page_invert", "drop_peaks", "add_threshold",
         "dark_peaks_fixed", "page_smooth")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "cd.npz")


def _kwargs(z, name):
    kw = json.loads(str(z[f"{name}_kwargs"]))
    if "methods" in kw:
        kw["methods"] = tuple(kw["methods"])
    return kw


@pytest.mark.parametrize("name", CASES)
def test_measure_cds_matches_reference_cpu(golden, name):
    from imageprocessor_new_b200 import measure_cds

    z = golden
    img = z[f"{name}_img"]
    kw = _kwargs(z, name)
    res = measure_cds(img, backend="gpu", **kw)
    if kw.get("seeds") == "peaks":
        # Peak positions come from the smoothed signal, whose width follows the pitch of an FFT
        # autocorrelation (cuFFT here, pocketfft in the reference): same seeds to 1e-9 px.
        assert res.meta["pitch_px"] == pytest.approx(float(z[f"{name}_pitch"]), rel=1e-9)
        assert res.seeds_xy.shape == z[f"{name}_seeds"].shape
        np.testing.assert_allclose(res.seeds_xy, z[f"{name}_seeds"], rtol=0, atol=1e-9)
    else:
        # Cells: seeds bit-exact.
        np.testing.assert_array_equal(res.seeds_xy, z[f"{name}_seeds"])
    np.testing.assert_array_equal(res.cell_labels, z[f"{name}_cell_labels"])
    # Deblending: same passes, outer iterations per pass, seeds added and dropped.
    meta = z[f"{name}_meta"]
    assert res.meta["deblend_iterations_used"] == meta[0]
    assert res.meta["deblend_passes"] == meta[1]
    assert res.meta["deblend_pass_iterations"] == list(z[f"{name}_passes"])
    assert res.meta["seeds_added_from_residual"] == meta[2]
    assert res.meta["seeds_dropped_as_insignificant"] == meta[3]
    assert res.meta["background_source"] == str(z[f"{name}_source"])
    np.testing.assert_allclose(res.deblend_model["params"], z[f"{name}_params"], rtol=0, atol=1e-6)
    for method in z[f"{name}_methods"]:
        method = str(method)
        got = res.measurements[method]
        status = z[f"{name}_{method}_status"]
        assert got.status.shape == status.shape, method
        if len(status):
            assert np.mean(got.status == status) >= 0.999, method
        both = got.valid & (status == "ok")
        cd = z[f"{name}_{method}_m_cd_equivalent_px"]
        delta = np.abs(got.metrics["cd_equivalent_px"][both] - cd[both])
        assert delta.max(initial=0) <= 2e-3, (method, delta.max(initial=0))
        centers = z[f"{name}_{method}_centers"]
        fin = np.isfinite(centers).all(axis=1) & np.isfinite(got.centers_xy).all(axis=1)
        assert np.abs(got.centers_xy[fin] - centers[fin]).max(initial=0) <= 1e-3, method


def _mixed_page(dtype):
    """288 x 288 page, 48 px pitch, holes of 30 and 12 px diameter alternating: the large holes'
    cell boxes are wider than 32 columns (the initial fit's per-pixel border test), the small ones'
    narrower (its row-mask path)."""
    from imageprocessor_new_b200 import synthetic

    rng = np.random.default_rng(7)
    shape = (288, 288)
    centers = synthetic.square_grid(shape, 48.0, rng)
    d = np.where(np.arange(len(centers)) % 2 == 0, 30.0, 12.0)
    clean = synthetic.render(shape, centers, d, 1.5, amplitude=3000.0, background=1000.0)
    img = synthetic.add_noise(clean, rng, read_noise=20.0)
    if dtype == np.uint8:
        return (img >> 5).astype(np.uint8)
    return img.astype(dtype)


@pytest.mark.parametrize("dtype", [np.uint16, np.uint8, np.float32, np.float64])
def test_measure_cds_wide_and_narrow_cells_match_oracle(dtype):
    from imageprocessor_new_b200 import measure_cds
    from oracle import cd as ocd

    img = _mixed_page(dtype)
    kw = dict(methods=("gaussian",), area_max=2000)
    res = measure_cds(img, backend="gpu", **kw)
    ref = ocd.measure_cds(img, **kw)
    np.testing.assert_array_equal(res.seeds_xy, ref["seeds"])
    assert len(ref["seeds"]) == 36
    if dtype in (np.uint16, np.uint8):
        # Cell boxes are the component boxes grown by pad = 3 on each side.
        from oracle import segment as osg

        binary = osg.binarize(img, osg.otsu_threshold(img), False)
        _, _, stats, _ = osg.label_components(binary, 8)
        box_w = stats[1:, 2] + 6
        assert (box_w > 32).any() and (box_w <= 32).any()
    np.testing.assert_allclose(res.deblend_model["params"], ref["params"], rtol=0, atol=1e-6)
    got = res.measurements["gaussian"]
    want = ref["measurements"]["gaussian"]
    assert np.array_equal(got.status, want["status"])
    a, b = got.metrics["cd_equivalent_px"], want["metrics"]["cd_equivalent_px"]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(a)
    assert ok.sum() >= 30 and np.abs(a[ok] - b[ok]).max() <= 2e-3


def test_measure_cds_fixed_background_level_matches_oracle():
    """A given background level replaces the cell-border percentile in the initial fits (both the
    narrow-box and the per-pixel border paths skip it) and fixes the background map."""
    from imageprocessor_new_b200 import measure_cds
    from oracle import cd as ocd

    img = _mixed_page(np.uint16)
    kw = dict(methods=("gaussian",), area_max=2000, background_level=1000.0)
    res = measure_cds(img, backend="gpu", **kw)
    ref = ocd.measure_cds(img, **kw)
    np.testing.assert_array_equal(res.seeds_xy, ref["seeds"])
    # FP64 sums in another order: amplitudes (~4000 counts) agree to 1e-9 relative, positions and
    # shapes to 1e-6 absolute.
    np.testing.assert_allclose(res.deblend_model["params"], ref["params"], rtol=1e-9, atol=1e-6)
    a = res.measurements["gaussian"].metrics["cd_equivalent_px"]
    b = ref["measurements"]["gaussian"]["metrics"]["cd_equivalent_px"]
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(a)
    assert ok.sum() >= 30 and np.abs(a[ok] - b[ok]).max() <= 2e-3
