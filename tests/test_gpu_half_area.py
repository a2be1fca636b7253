"""The half_area family on the GPU (subpx/_cpu/invariant_cd.py:551-875): half_area (median local
level), half_area_min (minimum level) and half_area_min_avg (minimum level, averaged peak).

Against the reference's own CPU measure_cds (golden fixtures, tests/golden/invariant.npz) through the
whole pipeline, and against the oracle's restatement on the GPU pipeline's own cleaned cells, which
isolates the kernel. The area is a count of 1/16 px^2 sub-pixels above a threshold and the outline a
search along rays in 1/8 px steps: decisions that agree when the enlargements agree to rounding.
"""

import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = ("staggered_half", "page_half", "lattice14_half")
HALF = ("half_area", "half_area_min", "half_area_min_avg")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "invariant.npz")


def _kwargs(z, name):
    kw = json.loads(str(z[f"{name}_kwargs"]))
    kw["methods"] = tuple(kw["methods"])
    return kw


def _close(a, b, frac=0.99, atol=1e-9, worst=None):
    """NaN where the other is NaN, and nearly every value within atol (all within `worst`)."""
    assert np.array_equal(np.isnan(a), np.isnan(b))
    ok = ~np.isnan(b)
    if not ok.any():
        return
    d = np.abs(a[ok] - b[ok])
    assert np.mean(d <= atol) >= frac, d.max()
    if worst is not None:
        assert d.max() <= worst, d.max()


@pytest.mark.parametrize("name", CASES)
def test_half_area_matches_reference_cpu(golden, name):
    from imageprocessor_new_b200 import measure_cds

    z = golden
    kw = _kwargs(z, name)
    res = measure_cds(z[f"{name}_img"], backend="gpu", **kw)
    assert list(res.measurements) == list(kw["methods"])
    for m in kw["methods"]:
        if m not in HALF:
            continue
        got = res.measurements[m]
        status = z[f"{name}_{m}_status"]
        assert np.mean(got.status == status) >= 0.99, m
        same = got.status == status
        for metric in ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "perimeter_px", "threshold",
                       "local_level", "mean_signal", "peak_signal"):
            ref = z[f"{name}_{m}_m_{metric}"]
            # Areas move by whole sub-pixels (1/16 px^2) where a sub-pixel sits on the threshold.
            _close(got.metrics[metric][same], ref[same], atol=1e-6 * max(1.0, np.nanmax(np.abs(ref), initial=0.0)),
                   worst=0.25 if "px" in metric else None)
        c, cz = got.centers_xy[same], z[f"{name}_{m}_centers"][same]
        _close(c.ravel(), cz.ravel(), atol=1e-9, worst=0.05)
        assert got.geometry["edge_px"].shape == z[f"{name}_{m}_edge_px"].shape
        _close(got.geometry["edge_px"][same].ravel(), z[f"{name}_{m}_edge_px"][same].ravel(), frac=0.98)


@pytest.mark.parametrize("name", ("staggered_half", "lattice14_half"))
def test_half_area_kernel_matches_oracle_on_same_cells(golden, name):
    """The GPU's cleaned cells through the oracle's half_area family: same statuses, areas and
    outlines in (nearly) every cell; metrics to rounding."""
    from imageprocessor_new_b200 import measure_cds
    from oracle import invariant as oi

    z = golden
    kw = _kwargs(z, name)
    kw["methods"] = HALF
    res = measure_cds(z[f"{name}_img"], backend="gpu", **kw)
    ref = oi.half_areas(res.rois, res.masks, res.origins_xy, 128, HALF)
    for m in HALF:
        got, want = res.measurements[m], ref[m]
        np.testing.assert_array_equal(got.status, want["status"], err_msg=m)
        for metric, v in want["metrics"].items():
            if metric == "background":
                continue
            _close(got.metrics[metric], v, frac=0.995, atol=1e-9 * max(1.0, np.nanmax(np.abs(v), initial=0.0)))
        _close(got.centers_xy.ravel(), want["centers"].ravel(), frac=0.995, atol=1e-9)
        _close(got.geometry["edge_px"].ravel(), want["edge_px"].ravel(), frac=0.99)


def test_half_area_options_and_shapes():
    from imageprocessor_new_b200 import measure_cds, synthetic

    page = synthetic.page_square(0).image[:256, :320]
    full = measure_cds(page, backend="gpu", methods=HALF, area_max=400)
    lean = measure_cds(page, backend="gpu", methods=HALF, area_max=400, metrics_only=True)
    bare = measure_cds(page, backend="gpu", methods=HALF, area_max=400, outlines=False)
    n = len(full.seeds_xy)
    for m in HALF:
        p, q, r = full.measurements[m], lean.measurements[m], bare.measurements[m]
        assert p.contours_xy.shape == (n, 129, 2) and p.geometry["edge_px"].shape == (n, 128)
        assert q.contours_xy.shape == (n, 0, 2) and q.geometry["edge_px"].shape == (n, 0)
        assert np.isnan(r.geometry["edge_px"]).all() and np.isnan(r.metrics["perimeter_px"]).all()
        for metric in p.metrics:
            if metric != "perimeter_px":
                np.testing.assert_array_equal(p.metrics[metric], q.metrics[metric])
                np.testing.assert_array_equal(p.metrics[metric], r.metrics[metric])
        assert list(p.metrics)[-3:] == ["local_level", "threshold", "mean_signal"]
    # A lower level takes more of the spot.
    low = measure_cds(page, backend="gpu", methods=("half_area",), area_max=400, half_area_level=0.3)
    ok = full.measurements["half_area"].valid & low.measurements["half_area"].valid
    assert ok.any()
    assert (low.measurements["half_area"].metrics["area_px2"][ok] > full.measurements["half_area"].metrics["area_px2"][ok]).all()
    with pytest.raises(ValueError):
        measure_cds(page, backend="gpu", methods=("half_area",), half_area_level=1.5)
