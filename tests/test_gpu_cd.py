"""measure_cds on the GPU against the reference's own CPU measure_cds (golden fixtures)."""

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = {
    "lattice2": dict(area_max=400),
    "lattice14": dict(area_max=400, methods=("gaussian", "halfmax")),
    "page": dict(area_max=400),
    "staggered": dict(area_max=400),
    "page_invert": dict(area_max=400, invert=True, methods=("gaussian", "logquad")),
}


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "cd.npz")


@pytest.mark.parametrize("name", list(CASES))
def test_measure_cds_matches_reference_cpu(golden, name):
    from imageprocessor_new_b200 import measure_cds

    z = golden
    img = z[f"{name}_img"]
    res = measure_cds(img, backend="gpu", **CASES[name])
    # Cells: seeds and Voronoi labels bit-exact.
    np.testing.assert_array_equal(res.seeds_xy, z[f"{name}_seeds"])
    np.testing.assert_array_equal(res.cell_labels, z[f"{name}_cell_labels"])
    # Deblending: same number of outer iterations and passes.
    meta = z[f"{name}_meta"]
    assert res.meta["deblend_iterations_used"] == meta[0]
    assert res.meta["deblend_passes"] == meta[1]
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
