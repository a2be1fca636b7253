"""The CPU oracle against the golden fixtures produced by the reference's own CPU path."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import centers as oc
from oracle import segment as osg
from oracle import voronoi as ov


def _load(name):
    return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)


def test_otsu_and_triangle_match_opencv():
    z = _load("thresholds")
    for i in range(int(z["n"])):
        img = z[f"img{i}"]
        assert osg.otsu_threshold(img) == z["otsu"][i], i
        if img.dtype == np.uint8:
            assert osg.triangle_threshold(img) == z["triangle"][i], i


@pytest.mark.parametrize("conn", [8, 4])
def test_ccl_numbering_and_stats_match_opencv(conn):
    z = _load("ccl")
    for i in range(int(z["n"])):
        shape = tuple(z[f"shape{i}"])
        mask = np.unpackbits(z[f"mask{i}"])[: shape[0] * shape[1]].reshape(shape).astype(bool)
        num, labels, stats, cents = osg.label_components(mask, conn)
        np.testing.assert_array_equal(labels, z[f"labels{i}_{conn}"])
        np.testing.assert_array_equal(stats[1:], z[f"stats{i}_{conn}"][1:])
        np.testing.assert_array_equal(cents[1:], z[f"cent{i}_{conn}"][1:])
        # Background row: area and bbox as OpenCV.
        np.testing.assert_array_equal(stats[0], z[f"stats{i}_{conn}"][0])


def test_detect_centers_match_reference_cpu():
    z = _load("centers")
    params = {"page": dict(threshold="otsu", area_max=400), "dots": dict(threshold="otsu", area_max=50),
              "small": dict(threshold="otsu", area_max=200), "dots_tri": dict(threshold="triangle", area_max=50),
              "small_morph": dict(threshold="otsu", area_max=200, morph_open=1, morph_close=1),
              "page_morph": dict(threshold="otsu", area_max=400, morph_open=2, morph_close=1)}
    for name in z["names"]:
        img = z[f"{name}_img"]
        for refine in ("weighted", "logquad", "edge_gradmoment", "none", "auto"):
            got = oc.detect_centers(img, refine_method=refine, **params[str(name)])
            want = z[f"{name}_{refine}"]
            assert got.shape == want.shape, (name, refine)
            tol = 1e-9 if refine in ("logquad", "auto") else 0.0
            np.testing.assert_allclose(got, want, rtol=0, atol=tol, err_msg=f"{name} {refine}")


def test_voronoi_labels_match_reference():
    z = _load("voronoi")
    for name in z["names"]:
        seeds, shape = z[f"{name}_seeds"], tuple(z[f"{name}_shape"])
        np.testing.assert_array_equal(ov.voronoi_labels(seeds, shape), z[f"{name}_labels"], err_msg=str(name))


def test_tiled_rules_match_reference():
    z = _load("tiled")
    got = oc.detect_tiled(z["img"], tile_h=int(z["tile_h"]), overlap=int(z["overlap"]), area_max=200,
                          refine_method="logquad")
    want = z["centers"]
    assert got.shape == want.shape
    key = lambda a: a[np.lexsort((a[:, 1], a[:, 0]))]
    np.testing.assert_allclose(key(got), key(want), rtol=0, atol=1e-9)


def _cd_kwargs(z, name):
    """measure_cds keyword arguments the fixture was made with (stored beside it as JSON)."""
    import json

    kw = json.loads(str(z[f"{name}_kwargs"]))
    if "methods" in kw:
        kw["methods"] = tuple(kw["methods"])
    return kw


# lattice14: seeds="peaks" on a pitch / FWHM 1.4 array; drop_peaks / add_threshold: seed revision
# dropping / adding seeds (two deblend passes); dark_peaks_fixed: inverted, fixed background level;
# page_smooth: smooth_sigma = 1 in the radial profiles.
@pytest.mark.parametrize("name", ["lattice2", "page", "page_invert", "lattice14", "drop_peaks", "add_threshold",
                                  "dark_peaks_fixed", "page_smooth"])
def test_measure_cds_oracle_matches_reference(name):
    from oracle import cd as ocd

    z = _load("cd")
    kw = _cd_kwargs(z, name)
    got = ocd.measure_cds(z[f"{name}_img"], **kw)
    np.testing.assert_array_equal(got["seeds"], z[f"{name}_seeds"])
    np.testing.assert_array_equal(got["cell_labels"], z[f"{name}_cell_labels"])
    assert got["iterations_used"] == z[f"{name}_meta"][0]
    assert got["passes"] == list(z[f"{name}_passes"])
    assert (got["added"], got["dropped"]) == tuple(z[f"{name}_meta"][2:4])
    np.testing.assert_allclose(got["params"], z[f"{name}_params"], rtol=0, atol=1e-9)
    for method in z[f"{name}_methods"]:
        method = str(method)
        r = got["measurements"][method]
        np.testing.assert_array_equal(r["status"], z[f"{name}_{method}_status"])
        np.testing.assert_allclose(r["metrics"]["cd_equivalent_px"], z[f"{name}_{method}_m_cd_equivalent_px"],
                                   rtol=0, atol=1e-9, equal_nan=True)
        np.testing.assert_allclose(r["contours"], z[f"{name}_{method}_contours"], rtol=0, atol=1e-9, equal_nan=True)


# The projection CD method (subpx/_cpu/invariant_cd.py:365-421) beside others: staggered and square
# pages, a lattice, an inverted page, and a dense peak-seeded lattice where most cells' steepest
# points reach the cell border (edge_at_cell_border); the half_area family (551-875) on a staggered
# page, a square page and the dense lattice (region_at_cell_border).
@pytest.mark.parametrize("name", ["staggered", "page", "lattice2", "page_invert", "lattice14", "staggered_half",
                                  "page_half", "lattice14_half"])
def test_projection_oracle_matches_reference(name):
    from oracle import cd as ocd

    z = _load("invariant")
    kw = _cd_kwargs(z, name)
    got = ocd.measure_cds(z[f"{name}_img"], **kw)
    np.testing.assert_array_equal(got["seeds"], z[f"{name}_seeds"])
    assert list(got["measurements"]) == [str(m) for m in z[f"{name}_methods"]]
    for method in z[f"{name}_methods"]:
        method = str(method)
        r = got["measurements"][method]
        np.testing.assert_array_equal(r["status"], z[f"{name}_{method}_status"])
        for metric, v in r["metrics"].items():
            np.testing.assert_array_equal(v, z[f"{name}_{method}_m_{metric}"], err_msg=f"{method} {metric}")
        np.testing.assert_array_equal(r["centers"], z[f"{name}_{method}_centers"])
        np.testing.assert_array_equal(r["contours"], z[f"{name}_{method}_contours"])
        if f"{name}_{method}_edge_px" in z.files:
            np.testing.assert_array_equal(r["edge_px"], z[f"{name}_{method}_edge_px"])


# The tail family (subpx/_cpu/invariant_cd.py:878-1068): windows of tail_window pitches holding each
# hole's share of the light, measured with the median of the territory's farthest tenth as the level
# (tail_area), none (tail_area_norm), the steepness-weighted mean (edge_area), the foot of the edge
# (foot_area) and the image's median foot ratio (foot_area_ratio); options on a square page, and a
# dense peak-seeded lattice.
@pytest.mark.parametrize("name", ["staggered_tail", "lattice2_tail", "page_tail", "lattice14_tail"])
def test_tail_oracle_matches_reference(name):
    import json

    from oracle import cd as ocd

    z = _load("tail")
    kw = _cd_kwargs(z, name)
    outlines = kw.pop("outlines", True)
    got = ocd.measure_cds(z[f"{name}_img"], **kw)
    np.testing.assert_array_equal(got["seeds"], z[f"{name}_seeds"])
    meta = json.loads(str(z[f"{name}_meta"]))
    assert got["tail_info"]["tail_window_px"] == meta["tail_window_px"]
    assert got["tail_info"].get("foot_ratio") == meta["foot_ratio"]
    for method in kw["methods"]:
        r = got["measurements"][method]
        np.testing.assert_array_equal(r["status"], z[f"{name}_{method}_status"])
        for metric, v in r["metrics"].items():
            if metric == "background" or (metric == "perimeter_px" and not outlines):
                continue
            np.testing.assert_array_equal(v, z[f"{name}_{method}_m_{metric}"], err_msg=f"{method} {metric}")
        np.testing.assert_array_equal(r["centers"], z[f"{name}_{method}_centers"])
        np.testing.assert_array_equal(r["center_local"], z[f"{name}_{method}_center_local"])
        if outlines:
            np.testing.assert_array_equal(r["edge_px"], z[f"{name}_{method}_edge_px"].astype(np.float64))


# The disk and flux_ratio methods (subpx/_cpu/invariant_cd.py:94-306, 1069-1206): the Airy-blurred,
# pixel-averaged disk table, the batched LM of each hole's disk, a second round with the neighbours
# re-rendered from the disk fits (near and far field), the blur given or calibrated by bisection on
# nominal_cd, the flux ratios with a dark level and scale.
@pytest.mark.parametrize("name", ["lattice_psf", "lattice_nominal", "staggered_disk"])
def test_disk_oracle_matches_reference(name):
    import json

    from oracle import cd as ocd

    z = _load("disk")
    kw = _cd_kwargs(z, name)
    got = ocd.measure_cds(z[f"{name}_img"], **kw)
    np.testing.assert_array_equal(got["seeds"], z[f"{name}_seeds"])
    meta = json.loads(str(z[f"{name}_meta"]))
    for key in ("psf_fwhm_px", "psf_source", "disk_median_cd_px", "flux_ratio_scale"):
        if meta.get(key) is not None:
            assert got["tail_info"][key] == meta[key], key
    for method in kw["methods"]:
        r = got["measurements"][method]
        np.testing.assert_array_equal(r["status"], z[f"{name}_{method}_status"])
        for metric, v in r["metrics"].items():
            if metric == "background":
                continue
            np.testing.assert_array_equal(v, z[f"{name}_{method}_m_{metric}"], err_msg=f"{method} {metric}")
        np.testing.assert_array_equal(r["centers"], z[f"{name}_{method}_centers"])
        np.testing.assert_array_equal(r["edge_px"], z[f"{name}_{method}_edge_px"])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_morphology_matches_opencv(seed):
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(seed)
    fg = rng.random((61, 83)) < (0.35 + 0.2 * seed)
    fg[0, :] = True        # borders: pixels outside must not erode or dilate anything
    fg[:, -1] = seed % 2 == 0
    bw = fg.astype(np.uint8) * 255
    k = cv2.getStructuringElement(cv2.MORPH_ELLIPSE, (3, 3))
    for o, c in ((1, 0), (0, 1), (2, 1), (1, 3)):
        want = bw
        if o:
            want = cv2.morphologyEx(want, cv2.MORPH_OPEN, k, iterations=o)
        if c:
            want = cv2.morphologyEx(want, cv2.MORPH_CLOSE, k, iterations=c)
        np.testing.assert_array_equal(osg.morphology(fg, o, c), want > 0, err_msg=f"open {o} close {c}")


@pytest.mark.parametrize("n", [0, 1, 300, 2000])
def test_pairwise_dedupe_equals_kdtree_dedupe(n):
    """The reference's O(N^2) dedupe loop and the oracle's KD-tree restatement give the same clusters
    (as sorted sets of means)."""
    rng = np.random.default_rng(n)
    base = rng.uniform(0, 300, (n, 2))
    pts = np.concatenate([base, base[: n // 3] + rng.normal(0, 0.6, (n // 3, 2))]) if n else np.zeros((0, 2))
    key = lambda a: a[np.lexsort((a[:, 1], a[:, 0]))]
    a, b = oc.dedupe(pts, 1.5), oc.dedupe_pairwise(pts, 1.5)
    assert a.shape == b.shape
    np.testing.assert_allclose(key(a), key(b), rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["page", "lattice"])
def test_model_background_centres_match_reference(name):
    """detect_centers(background="model"): centres re-refined on deblended cells (reference CPU path,
    tests/golden/centers_model.npz)."""
    z = _load("centers_model")
    for refine in ("weighted", "logquad", "none"):
        got, state, _ = oc.detect_centers_model(z[f"{name}_img"], refine_method=refine, threshold="otsu",
                                                area_max=400)
        np.testing.assert_allclose(got, z[f"{name}_{refine}"], rtol=0, atol=1e-9)
        assert state.iterations == int(z[f"{name}_{refine}_used"])
