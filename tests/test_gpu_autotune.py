"""The autotuner's knobs change launch shapes only: every setting gives bit-identical fits and
model images, and the tuner picks one of the candidates."""

import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_knobs_roundtrip_and_reject_bad_values():
    from imageprocessor_new_b200 import _lib, autotune

    before = autotune.current()
    try:
        for knob, values in autotune.KNOBS.items():
            for v in values:
                autotune.set(knob, v)
                assert autotune.get(knob) == v
        with pytest.raises(_lib.LibraryError):
            autotune.set("fit_warps", 3)
        with pytest.raises(_lib.LibraryError):
            autotune.set("no_such_knob", 1)
    finally:
        autotune.apply(before)


def test_every_setting_gives_identical_results(tmp_path, monkeypatch):
    import torch

    from imageprocessor_new_b200 import autotune, synthetic
    from imageprocessor_new_b200.deblend import Deblender
    from imageprocessor_new_b200.warmstart import page_cells

    before = autotune.current()
    page = torch.from_numpy(synthetic.page_staggered(1, shape=(1024, 1280)).image).cuda()
    cells = page_cells(page)
    outs = []
    try:
        for fw, fb, rt in itertools.product((2, 4, 8), (4, 16), (16, 32, 64)):
            autotune.apply({"fit_warps": fw, "fit_blocks_per_sm": fb, "render_tile": rt})
            dbl = Deblender(page, 1.0, cells)
            p, st, it = dbl.initial(dbl.max_iter)
            model = dbl.render(p)
            bg, _ = dbl.background_of(model, dbl.stats(p, st))
            q, st2, _, _ = dbl.iteration(p, model, bg)
            outs.append([a.cpu().numpy() for a in (p, st, it, model, q, st2)])
        for o in outs[1:]:
            for a, b in zip(outs[0], o):
                np.testing.assert_array_equal(a, b)
        monkeypatch.setenv("SPX_TUNE_CACHE", str(tmp_path / "tune.json"))
        res = autotune.tune(page, repeats=1)
        for knob, values in autotune.KNOBS.items():
            assert res["config"][knob] in values
        assert (tmp_path / "tune.json").exists()
        again = autotune.tune(page, repeats=1)   # from the cache
        assert again["config"] == res["config"]
    finally:
        autotune.apply(before)


def test_radial_ray_mappings_give_identical_cds():
    """One ray per thread with the spline window cached or read at every sample: the same edges,
    statuses and metrics bit for bit, with and without profile smoothing."""
    from imageprocessor_new_b200 import autotune, measure_cds, synthetic

    before = autotune.current()
    page = synthetic.page_staggered(2, shape=(768, 1024)).image
    try:
        for smooth in (0.0, 1.0):
            res = []
            for mode in (0, 2):
                autotune.set("radial_rays", mode)
                res.append(measure_cds(page, backend="gpu", methods=("gradient", "halfmax"), area_max=400,
                                       smooth_sigma=smooth))
            for other in res[1:]:
                for m in ("gradient", "halfmax"):
                    a, b = res[0].measurements[m], other.measurements[m]
                    np.testing.assert_array_equal(a.geometry["edge_px"], b.geometry["edge_px"])
                    np.testing.assert_array_equal(a.status, b.status)
                    np.testing.assert_array_equal(a.contours_xy, b.contours_xy)
                    for k in a.metrics:
                        np.testing.assert_array_equal(a.metrics[k], b.metrics[k], err_msg=k)
    finally:
        autotune.apply(before)
