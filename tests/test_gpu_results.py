"""Compact result files rebuilt on the device: a compact folder written by the reference's own
save_cd_results loads to the same arrays as its full folder (contours, measured cells, component
labels and background map rebuilt by spx_rebuild_contours / spx_clean_masked / the CCL / the tile
rows), and a compact folder of this package's own measure_cds result loads back to that result."""

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_reference_compact_folder_rebuilds_its_full_arrays():
    from imageprocessor_new_b200.results import load_cd_results

    full = load_cd_results(GOLDEN / "results_full")
    comp = load_cd_results(GOLDEN / "results_compact")
    np.testing.assert_array_equal(comp.component_labels, full.component_labels)
    np.testing.assert_allclose(comp.background_map, full.background_map, rtol=0, atol=1e-9)
    # The reference rebuilt its rois with NumPy; here the device's exp: agreement to rounding.
    scale = np.abs(full.rois).max()
    np.testing.assert_allclose(comp.rois, full.rois, rtol=0, atol=1e-12 * scale)
    for m in full.measurements:
        a, b = comp.measurements[m].contours_xy, full.measurements[m].contours_xy
        assert np.array_equal(np.isnan(a), np.isnan(b)), m
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9, err_msg=m)


@pytest.mark.parametrize("methods", [("gaussian", "logquad", "gradient", "halfmax")])
def test_own_compact_export_round_trip(tmp_path, methods):
    from imageprocessor_new_b200 import measure_cds, synthetic
    from imageprocessor_new_b200.results import load_cd_results, save_cd_results

    page = np.ascontiguousarray(synthetic.page_square(3).image[:200, :260])
    res = measure_cds(page, backend="gpu", methods=methods, area_max=400)
    save_cd_results(res, tmp_path / "c", compact=True)
    back = load_cd_results(tmp_path / "c")
    np.testing.assert_array_equal(back.component_labels, res.component_labels)
    np.testing.assert_array_equal(back.background_map, res.background_map)
    np.testing.assert_array_equal(back.rois, res.rois)  # same kernels' arithmetic
    for m in methods:
        a, b = back.measurements[m].contours_xy, res.measurements[m].contours_xy
        np.testing.assert_array_equal(a, b, err_msg=m)
        np.testing.assert_array_equal(back.measurements[m].metrics["cd_equivalent_px"],
                                      res.measurements[m].metrics["cd_equivalent_px"])


def test_compact_round_trip_area_methods(tmp_path):
    """Compact files of the projection, half_area and tail methods: contours rebuilt from center_local,
    edge_px and the cell origins (as the reference's loader rebuilds them). The measuring kernels
    draw projection's ellipse and the tail outlines (on windows around the holes, center_local then
    relative to the hole's cell) with other roundings, so the rebuilt vertices agree to 1e-9 px;
    metrics and statuses are unchanged."""
    from imageprocessor_new_b200 import measure_cds, synthetic
    from imageprocessor_new_b200.results import load_cd_results, save_cd_results

    methods = ("projection", "half_area_min_avg", "tail_area", "foot_area", "foot_area_ratio")
    page = np.ascontiguousarray(synthetic.page_square(3).image[:200, :260])
    # tail_window 0.8: windows of 53 px on this page (pitch about 32 px; the kernel takes up to 64 px).
    res = measure_cds(page, backend="gpu", methods=methods, area_max=400, tail_window=0.8)
    save_cd_results(res, tmp_path / "c", compact=True)
    back = load_cd_results(tmp_path / "c")
    for m in methods:
        a, b = back.measurements[m].contours_xy, res.measurements[m].contours_xy
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9, equal_nan=True, err_msg=m)
        for metric, v in res.measurements[m].metrics.items():
            np.testing.assert_array_equal(back.measurements[m].metrics[metric], v, err_msg=f"{m} {metric}")
        np.testing.assert_array_equal(back.measurements[m].status, res.measurements[m].status)
