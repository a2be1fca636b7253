"""detect_centers through the CUDA path against the reference CPU golden outputs and the oracle."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import centers as oc

pytestmark = pytest.mark.gpu

PARAMS = {"page": dict(threshold="otsu", area_max=400), "dots": dict(threshold="otsu", area_max=50),
          "small": dict(threshold="otsu", area_max=200), "dots_tri": dict(threshold="triangle", area_max=50),
          "small_morph": dict(threshold="otsu", area_max=200, morph_open=1, morph_close=1),
          "page_morph": dict(threshold="otsu", area_max=400, morph_open=2, morph_close=1)}


@pytest.mark.parametrize("refine", ["weighted", "logquad", "edge_gradmoment", "none", "auto"])
def test_detect_centers_matches_reference_cpu(refine):
    from imageprocessor_new_b200 import detect_centers

    z = np.load(GOLDEN / "centers.npz")
    for name in z["names"]:
        img = z[f"{name}_img"]
        got = detect_centers(img, backend="gpu", refine=refine, **PARAMS[str(name)])
        want = z[f"{name}_{refine}"]
        assert got.backend == "gpu"
        assert got.centers_xy.shape == want.shape, (name, refine)
        # weighted / none are exact on integer images; logquad solves normal equations and the edge
        # moments use pow(d, 8), whose last bit may differ from the host libm.
        tol = 1e-9 if refine in ("logquad", "auto", "edge_gradmoment") else 0.0
        np.testing.assert_allclose(got.centers_xy, want, rtol=0, atol=tol, err_msg=f"{name} {refine}")


@pytest.mark.parametrize("refine", ["weighted", "logquad", "edge_gradmoment"])
def test_detect_centers_page_against_oracle(refine):
    from imageprocessor_new_b200 import detect_centers, synthetic

    page = synthetic.page_square(3).image
    got = detect_centers(page, backend="gpu", threshold="otsu", refine=refine, area_max=400).centers_xy
    want = oc.detect_centers(page, threshold="otsu", refine_method=refine, area_max=400)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, rtol=0, atol=0.0 if refine == "weighted" else 1e-9)


def test_detect_centers_invert_and_edges():
    from imageprocessor_new_b200 import detect_centers, synthetic

    page = synthetic.page_square(4).image
    dark = (np.iinfo(np.uint16).max - page).astype(np.uint16)
    got = detect_centers(dark, backend="gpu", threshold="otsu", invert=True, refine="weighted", area_max=400)
    want = oc.detect_centers(dark, threshold="otsu", invert=True, refine_method="weighted", area_max=400)
    assert got.centers_xy.shape == want.shape
    np.testing.assert_array_equal(got.centers_xy, want)
    # A blob cut by the image border.
    crop = np.ascontiguousarray(page[5:300, 9:333])
    for refine in ("weighted", "edge_gradmoment", "logquad"):
        got = detect_centers(crop, backend="gpu", threshold="otsu", refine=refine, area_max=400).centers_xy
        want = oc.detect_centers(crop, threshold="otsu", refine_method=refine, area_max=400)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)


def test_empty_image_has_no_centers():
    from imageprocessor_new_b200 import detect_centers

    img = np.zeros((64, 80), np.uint16)
    res = detect_centers(img, backend="gpu", threshold="otsu")
    assert res.centers_xy.shape == (0, 2)


def test_bad_arguments_raise():
    from imageprocessor_new_b200 import detect_centers

    img = np.zeros((16, 16), np.uint16)
    with pytest.raises(ValueError):
        detect_centers(img, backend="gpu", refine="bogus")
    with pytest.raises(ValueError):
        detect_centers(img, backend="cpu")
    with pytest.raises(ValueError):
        detect_centers(np.zeros((4, 4, 3), np.uint8), backend="gpu")


def test_morphology_masks_match_oracle():
    import torch

    from imageprocessor_new_b200 import _lib, synthetic

    page = synthetic.page_square(2).image[:300, :417]
    thr = 2200.0
    fg = page > thr
    img_d = torch.from_numpy(np.ascontiguousarray(page)).cuda()
    h, w = page.shape
    stream = torch.cuda.current_stream().cuda_stream
    for o, c in ((1, 0), (0, 2), (2, 1), (3, 3)):
        bw = torch.empty((h, w), dtype=torch.uint8, device="cuda")
        tmp = torch.empty_like(bw)
        _lib.call("spx_binarize", img_d.data_ptr(), 1, h, w, None, thr, 0, bw.data_ptr(), stream)
        _lib.call("spx_morphology", bw.data_ptr(), h, w, o, c, tmp.data_ptr(), stream)
        from oracle import segment as osg

        want = osg.morphology(fg, o, c).astype(np.uint8) * 255
        np.testing.assert_array_equal(bw.cpu().numpy(), want, err_msg=f"open {o} close {c}")


def test_tiled_with_morphology_matches_untiled_rules():
    from imageprocessor_new_b200 import detect_centers, synthetic

    page = synthetic.page_square(1).image
    kw = dict(backend="gpu", threshold="otsu", refine="weighted", area_max=400, morph_open=1, morph_close=1)
    whole = detect_centers(page, tile_h=page.shape[0], overlap=0, **kw).centers_xy
    tiled = detect_centers(page, tile_h=300, overlap=64, **kw).centers_xy
    # Bands see the same global threshold; holes away from band edges are found identically.
    d = np.sqrt(((whole[:, None, :] - tiled[None, :, :]) ** 2).sum(-1)).min(axis=1)
    assert len(tiled) == len(whole)
    assert np.median(d) == 0.0


@pytest.mark.parametrize("name", ["page", "lattice"])
@pytest.mark.parametrize("refine", ["weighted", "logquad", "none"])
def test_model_background_refinement_matches_reference(name, refine):
    """detect_centers(background="model") on the GPU against the reference's CPU path (golden): the
    same centres to 1e-6 px (deblended cells in FP64, sums in another order) and deblend iterations."""
    from imageprocessor_new_b200 import detect_centers

    z = np.load(GOLDEN / "centers_model.npz")
    res = detect_centers(z[f"{name}_img"], backend="gpu", threshold="otsu", area_max=400, refine=refine,
                         background="model")
    want = z[f"{name}_{refine}"]
    assert res.centers_xy.shape == want.shape
    np.testing.assert_allclose(res.centers_xy, want, rtol=0, atol=1e-6)
    assert res.meta["deblend_iterations_used"] == int(z[f"{name}_{refine}_used"])
    assert res.meta["background"] == "model"
