"""The tail CD family on the GPU (subpx/_cpu/invariant_cd.py:878-1068): windows of tail_window pitches
holding each hole's share of the light (spx_wide_cells) measured with the five threshold rules
(spx_tail_area_cd).

Against the reference's own CPU measure_cds (golden fixtures, tests/golden/tail.npz) through the whole
pipeline; against the oracle's restatement fed with the GPU's own fitted models (a fixed background
level, so both sides hold the same map), which isolates the windows and the kernel; and the grid
neighbour search against a k-d tree. Areas are counts of 1/16 px^2 sub-pixels above a threshold and
outlines searches in 1/8 px steps: decisions that agree when the enlargements agree to rounding.
"""

import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TAIL = ("tail_area", "tail_area_norm", "edge_area", "foot_area", "foot_area_ratio")
CASES = ("staggered_tail", "lattice2_tail", "page_tail", "lattice14_tail")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN / "tail.npz")


def _kwargs(z, name):
    kw = json.loads(str(z[f"{name}_kwargs"]))
    kw["methods"] = tuple(kw["methods"])
    return kw


def _close(a, b, frac=0.99, atol=1e-9, worst=None):
    """NaN where the other is NaN (nearly everywhere), and nearly every value within atol."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert np.mean(np.isnan(a) == np.isnan(b)) >= frac
    ok = ~np.isnan(a) & ~np.isnan(b)
    if not ok.any():
        return
    d = np.abs(a[ok] - b[ok])
    assert np.mean(d <= atol) >= frac, d.max()
    if worst is not None:
        assert d.max() <= worst, d.max()


@pytest.mark.parametrize("name", CASES)
def test_tail_matches_reference_cpu(golden, name):
    from imageprocessor_new_b200 import measure_cds

    z = golden
    kw = _kwargs(z, name)
    outlines = kw.get("outlines", True)
    res = measure_cds(z[f"{name}_img"], backend="gpu", **kw)
    assert list(res.measurements) == list(kw["methods"])
    meta = json.loads(str(z[f"{name}_meta"]))
    assert res.meta["tail_window_px"] == meta["tail_window_px"]
    if meta.get("foot_ratio") is not None:
        assert abs(res.meta["foot_ratio"] - meta["foot_ratio"]) <= 1e-3 * abs(meta["foot_ratio"])
    for m in kw["methods"]:
        if m not in TAIL:
            continue
        got = res.measurements[m]
        status = z[f"{name}_{m}_status"]
        assert np.mean(got.status == status) >= 0.97, (m, np.unique(got.status, return_counts=True))
        same = got.status == status
        for metric in ("area_px2", "cd_equivalent_px", "cd_x_px", "cd_y_px", "threshold", "local_level",
                       "mean_signal", "peak_signal") + (("steepest_level",) if m == "foot_area" else ()):
            ref = z[f"{name}_{m}_m_{metric}"]
            scale = max(1.0, np.nanmax(np.abs(ref), initial=0.0))
            # Areas move by whole sub-pixels (1/16 px^2) where a sub-pixel sits on the threshold; the
            # fitted models (hence each window's share of the light) agree with the reference to 1e-6.
            _close(got.metrics[metric][same], ref[same], frac=0.95, atol=1e-4 * scale,
                   worst=1.0 if "px" in metric else None)
        _close(got.centers_xy[same].ravel(), z[f"{name}_{m}_centers"][same].ravel(), frac=0.95, atol=1e-4, worst=0.1)
        _close(got.geometry["center_local"][same].ravel(), z[f"{name}_{m}_center_local"][same].ravel(), frac=0.95,
               atol=1e-4, worst=0.1)
        if outlines:
            assert got.geometry["edge_px"].shape == z[f"{name}_{m}_edge_px"].shape
            _close(got.geometry["edge_px"][same].ravel(), z[f"{name}_{m}_edge_px"][same].ravel(), frac=0.97)
        else:
            assert np.isnan(got.metrics["perimeter_px"]).all()


@pytest.mark.parametrize("name", ("staggered_tail", "lattice2_tail"))
def test_tail_kernel_matches_oracle_on_same_models(golden, name):
    """The GPU run's fitted models through the oracle's windows and tail family (fixed background
    level): same statuses and outlines in (nearly) every window, metrics to rounding."""
    from imageprocessor_new_b200 import measure_cds
    from oracle import deblend as odb
    from oracle import invariant as oi

    z = golden
    kw = _kwargs(z, name)
    kw["methods"] = TAIL
    img = z[f"{name}_img"]
    level = float(np.percentile(img, 10))
    res = measure_cds(img, backend="gpu", background_level=level, **kw)
    dm = res.deblend_model
    params, report = dm["params"], dm["report"]
    hm, wm = res.meta["cell_stack_shape"]
    signal = img.astype(np.float64)
    state = odb.State.__new__(odb.State)
    state.params = params
    state.background_map = np.full(img.shape, level)
    state.model_image = odb.render(params, img.shape, max(hm, wm))
    masks = np.zeros((len(params), hm, wm), bool)
    origins = np.zeros((len(params), 2))
    want = oi.tail_areas(signal, state, masks, origins, report, 128, TAIL, pitch=res.meta["pitch_px"])
    assert res.meta["tail_window_px"] == want["_info"]["tail_window_px"]
    for m in TAIL:
        got, ref = res.measurements[m], want[m]
        assert np.mean(got.status == ref["status"]) >= 0.99, m
        same = got.status == ref["status"]
        for metric, v in ref["metrics"].items():
            if metric == "background":
                continue
            scale = max(1.0, np.nanmax(np.abs(v), initial=0.0))
            _close(got.metrics[metric][same], v[same], frac=0.99, atol=1e-7 * scale)
        _close(got.centers_xy[same].ravel(), ref["centers"][same].ravel(), frac=0.99, atol=1e-7)
        _close(got.geometry["edge_px"][same].ravel(), ref["edge_px"][same].ravel(), frac=0.99)


@pytest.mark.parametrize("case", ["random", "duplicates", "lattice"])
def test_window_neighbours_match_kdtree(case):
    """spx_wide_cells' 8 nearest holes per reported hole against scipy's k-d tree (distance ties, as on
    a lattice, may order equal distances differently: compared as distance lists)."""
    import torch
    from scipy.spatial import cKDTree

    from imageprocessor_new_b200 import _device as dev
    from imageprocessor_new_b200 import _lib

    rng = np.random.default_rng(3)
    h, w = 300, 400
    if case == "lattice":
        yy, xx = np.mgrid[10:290:14, 10:390:14]
        centers = np.column_stack((xx.ravel(), yy.ravel())).astype(float)
    else:
        centers = rng.uniform([0, 0], [w, h], size=(700, 2))
        if case == "duplicates":
            centers[350:400] = centers[:50]
    n = len(centers)
    params = np.zeros((n, 6))
    params[:, 0] = 1.0
    params[:, 1:3] = centers - np.floor(centers)  # ROI-local centres in boxes at the integer parts
    boxes = np.column_stack((np.floor(centers), np.full((n, 2), 8))).astype(np.int32)
    report = np.arange(0, n, 3, dtype=np.int32)
    img = torch.zeros((h, w), dtype=torch.float64, device="cuda")
    model = torch.zeros((h, w), dtype=torch.float64, device="cuda")
    bg = _lib.BgMap(None, None, None, 1, w, 0.0, _lib.BG_FIXED)
    radius, side = 3, 7
    m = len(report)
    outs = [dev.empty((m, side, side), t) for t in (torch.float32, torch.uint8, torch.uint8, torch.uint8)]
    org = dev.empty((m, 2), torch.int32)
    nb = dev.empty((m, 9), torch.int32)
    ws = dev.workspace(_lib.size("spx_wide_cells_workspace_bytes", n, m, h, w, 14.0))
    # The uploads stay referenced until the kernels have read them (the copies and launches are asynchronous).
    params_d, boxes_d, report_d = dev.upload(params), dev.upload(boxes), dev.upload(report)
    _lib.call("spx_wide_cells", img.data_ptr(), 3, 1.0, h, w, bg, model.data_ptr(), params_d.data_ptr(),
              boxes_d.data_ptr(), n, 8, 8, report_d.data_ptr(), m, radius, 14.0, 1e-3,
              *(o.data_ptr() for o in outs), org.data_ptr(), nb.data_ptr(), ws.data_ptr(), ws.numel(),
              dev.stream_ptr())
    got = nb.cpu().numpy()
    glob = params[:, 1:3] + boxes[:, :2]
    assert (got[:, 0] == report).all()
    d_ref, i_ref = cKDTree(glob).query(glob[report], k=10)
    for r in range(m):
        others = [j for j in got[r, 1:]]
        assert -1 not in others and report[r] not in others
        d_got = np.sort(np.hypot(*(glob[others] - glob[report[r]]).T))
        # the k-d tree's 9 nearest besides the hole itself (it may list the hole itself or a duplicate first)
        cand = [(d, j) for d, j in zip(d_ref[r], i_ref[r]) if j != report[r]][:8]
        np.testing.assert_allclose(d_got, np.sort([d for d, _ in cand]), rtol=0, atol=1e-9)
    np.testing.assert_array_equal(org.cpu().numpy(), np.rint(glob[report]).astype(np.int64) - radius)


def test_tail_few_holes_and_options():
    """Fewer modelled holes than the 8 neighbours a window looks at (the reference's k-d tree query
    then asks for fewer), against the oracle on the same models; the reference's argument checks;
    windows wider than the kernel's 64 px refused; a page without holes gives empty results."""
    from imageprocessor_new_b200 import measure_cds, synthetic
    from oracle import deblend as odb
    from oracle import invariant as oi

    img, _ = synthetic.gaussian_lattice(2.0, shape=(40, 60), seed=0)  # 8 holes, windows past the edges
    level = float(np.percentile(img, 10))
    res = measure_cds(img, backend="gpu", methods=TAIL, area_max=400, background_level=level)
    dm = res.deblend_model
    params, report = dm["params"], dm["report"]
    assert 1 < len(params) <= 8
    hm, wm = res.meta["cell_stack_shape"]
    state = odb.State.__new__(odb.State)
    state.params = params
    state.background_map = np.full(img.shape, level)
    state.model_image = odb.render(params, img.shape, max(hm, wm))
    want = oi.tail_areas(img.astype(np.float64), state, np.zeros((len(params), hm, wm), bool),
                         np.zeros((len(params), 2)), report, 128, TAIL, pitch=res.meta["pitch_px"])
    for m in TAIL:
        np.testing.assert_array_equal(res.measurements[m].status, want[m]["status"], err_msg=m)
        _close(res.measurements[m].metrics["area_px2"], want[m]["metrics"]["area_px2"], frac=1.0, atol=1e-9)
    with pytest.raises(ValueError, match="tail_area_level"):
        measure_cds(img, backend="gpu", methods=("tail_area",), tail_area_level=1.0)
    with pytest.raises(ValueError, match="tail_window"):
        measure_cds(img, backend="gpu", methods=("tail_area",), tail_window=2.5)
    page = synthetic.page_staggered(0, shape=(256, 256)).image
    with pytest.raises(NotImplementedError, match="64 px"):
        measure_cds(page, backend="gpu", methods=("tail_area",), area_max=400, tail_window=1.5)
    empty = measure_cds(np.full((64, 64), 1000, np.uint16), backend="gpu", methods=TAIL)
    for m in TAIL:
        assert len(empty.measurements[m].status) == 0
        assert "steepest_level" in empty.measurements[m].metrics or m != "foot_area"
