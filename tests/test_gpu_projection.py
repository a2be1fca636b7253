"""The projection CD method on the GPU (subpx/_cpu/invariant_cd.py:365-421).

Against the reference's own CPU measure_cds (golden fixtures, tests/golden/invariant.npz) through
the whole pipeline, and against the oracle's restatement on the GPU pipeline's own cleaned cells,
which isolates the kernel: the widths are grid decisions (0.02 px steps of the profile splines),
identical when the splines agree to rounding.
"""

import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = ("staggered", "page", "lattice2", "page_invert", "lattice14")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "invariant.npz")


def _kwargs(z, name):
    kw = json.loads(str(z[f"{name}_kwargs"]))
    kw["methods"] = tuple(kw["methods"])
    return kw


@pytest.mark.parametrize("name", CASES)
def test_projection_matches_reference_cpu(golden, name):
    from imageprocessor_new_b200 import measure_cds

    z = golden
    kw = _kwargs(z, name)
    res = measure_cds(z[f"{name}_img"], backend="gpu", **kw)
    assert list(res.measurements) == list(kw["methods"])
    if kw.get("seeds") == "peaks":
        np.testing.assert_allclose(res.seeds_xy, z[f"{name}_seeds"], rtol=0, atol=1e-9)
    else:
        np.testing.assert_array_equal(res.seeds_xy, z[f"{name}_seeds"])
    got = res.measurements["projection"]
    status = z[f"{name}_projection_status"]
    np.testing.assert_array_equal(got.status, status)
    assert got.valid.tolist() == (status == "ok").tolist()
    for metric in ("cd_x_px", "cd_y_px", "cd_equivalent_px", "area_px2", "perimeter_px"):
        a, b = got.metrics[metric], z[f"{name}_projection_m_{metric}"]
        assert np.array_equal(np.isnan(a), np.isnan(b)), metric
        ok = ~np.isnan(b)
        # Same grid decisions in (almost) every cell: a width moves by whole 0.02 px steps.
        assert np.mean(np.abs(a[ok] - b[ok]) <= 1e-9) >= 0.99, metric
        assert np.abs(a[ok] - b[ok]).max(initial=0) <= 0.1, metric
    np.testing.assert_allclose(got.metrics["peak_signal"], z[f"{name}_projection_m_peak_signal"], rtol=1e-7,
                               atol=1e-6)
    c, cz = got.centers_xy, z[f"{name}_projection_centers"]
    assert np.array_equal(np.isfinite(c), np.isfinite(cz))
    fin = np.isfinite(cz).all(axis=1)
    assert np.mean(np.abs(c[fin] - cz[fin]).max(axis=1) <= 1e-9) >= 0.99
    assert got.contours_xy.shape == z[f"{name}_projection_contours"].shape
    assert got.geometry["edge_px"].shape == z[f"{name}_projection_edge_px"].shape


@pytest.mark.parametrize("name", ("staggered", "lattice14"))
def test_projection_kernel_matches_oracle_on_same_cells(golden, name):
    """The GPU's cleaned cells through the oracle's projection: the same decisions, widths and
    centres bit for bit, contours and edge radii to rounding (cos / sin of the ray angles)."""
    from imageprocessor_new_b200 import measure_cds
    from oracle import invariant as oi

    z = golden
    kw = _kwargs(z, name)
    kw["methods"] = ("projection",)
    res = measure_cds(z[f"{name}_img"], backend="gpu", **kw)
    got = res.measurements["projection"]
    ref = oi.projection(res.rois, res.masks, res.origins_xy, 128)
    np.testing.assert_array_equal(got.status, ref["status"])
    for metric in ("cd_x_px", "cd_y_px", "cd_equivalent_px", "area_px2", "perimeter_px", "peak_signal"):
        np.testing.assert_array_equal(got.metrics[metric], ref["metrics"][metric], err_msg=metric)
    np.testing.assert_array_equal(got.centers_xy, ref["centers"])
    np.testing.assert_array_equal(got.geometry["center_local"], ref["center_local"])
    np.testing.assert_allclose(got.geometry["edge_px"], ref["edge_px"], rtol=1e-14, atol=0, equal_nan=True)
    np.testing.assert_allclose(got.contours_xy, ref["contours"], rtol=0, atol=1e-11, equal_nan=True)


def test_projection_metrics_only_and_summary():
    from imageprocessor_new_b200 import measure_cds, synthetic

    page = synthetic.page_square(0).image[:256, :320]
    full = measure_cds(page, backend="gpu", methods=("projection", "halfmax"), area_max=400)
    lean = measure_cds(page, backend="gpu", methods=("projection", "halfmax"), area_max=400, metrics_only=True)
    summ = measure_cds(page, backend="gpu", methods=("projection",), area_max=400, summary_only=True)
    n = len(full.seeds_xy)
    p, q = full.measurements["projection"], lean.measurements["projection"]
    assert p.contours_xy.shape == (n, 129, 2) and p.geometry["edge_px"].shape == (n, 128)
    assert q.contours_xy.shape == (n, 0, 2) and q.geometry["edge_px"].shape == (n, 0)
    for metric in p.metrics:
        np.testing.assert_array_equal(p.metrics[metric], q.metrics[metric])
        np.testing.assert_array_equal(p.metrics[metric], summ.measurements["projection"].metrics[metric])
    np.testing.assert_array_equal(p.status, summ.measurements["projection"].status)
    assert np.isfinite(p.metrics["background"]).all()
