"""Uneven stacks (imageprocessor_new_b200.stack): every cell of every image fitted in one launch.

Four 768 x 768 synthetic images with their own pitch, hole size, blur and noise. The one-launch
stack fits must be the per-image fits cell for cell (plain and warm-started), and per image the
plain fits of a sample of cells are checked against the FP64 oracle's initial fit
(oracle/deblend.py, restating subpx/_cpu/deblend.py:152-171 and 174-254 with the cell-border
10th percentile of :480-481).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stack():
    from imageprocessor_new_b200 import stack as st

    s = st.synth_stack(4, 768, seed=3)
    return s, st.stack_cells(s)


def _host(fits):
    return [t.cpu().numpy() for t in fits]


def test_stack_cells_are_the_per_image_cells(stack):
    from imageprocessor_new_b200 import warmstart as ws

    s, sc = stack
    counts = np.diff(sc.starts)
    assert len(set(counts.tolist())) > 1  # uneven
    for i in range(sc.images):
        c = ws.page_cells(s[i])
        sl = sc.image_of(i)
        assert c.n == counts[i]
        np.testing.assert_array_equal(sc.cells.rows[sl, :4] - [0, i * 768, 0, 0], c.rows[:, :4])
        b = sc.cells.boxes[sl].cpu().numpy()
        np.testing.assert_array_equal(b - [0, i * 768, 0, 0], c.boxes.cpu().numpy())
        vor = sc.cells.voronoi[i * 768:(i + 1) * 768].cpu().numpy()
        np.testing.assert_array_equal(vor - sc.starts[i], c.voronoi.cpu().numpy())


@pytest.mark.parametrize("warm", [False, True])
def test_one_launch_equals_per_image_fits(stack, warm):
    from imageprocessor_new_b200 import stack as st
    from imageprocessor_new_b200 import warmstart as ws

    s, sc = stack
    net = ws.WarmStartNet.load() if warm else None
    whole = _host(st.initial_fits(s, sc, net=net))
    for i in range(sc.images):
        c = ws.page_cells(s[i])
        w = None
        if warm:
            w = ws.predict_init(net, s[i], 1.0, c.seeds_d, c.boxes, c.n)
        part = _host(ws.initial_fits(s[i], c, warm=w, cost_tol=net.cost_tol if warm else 1e-12))
        sl = sc.image_of(i)
        for a, b in zip(whole, part):
            np.testing.assert_array_equal(a[sl], b)
    if warm:
        plain = _host(st.initial_fits(s, sc))
        ok = (whole[1] == 0) & (plain[1] == 0)
        assert ok.mean() > 0.95
        assert np.abs(whole[0][ok, 1:3] - plain[0][ok, 1:3]).max() <= 1e-3
        assert whole[2].mean() < plain[2].mean()


def test_stack_fits_against_fp64_oracle_per_image(stack):
    from scipy.ndimage import binary_erosion

    from imageprocessor_new_b200 import _lib
    from imageprocessor_new_b200 import stack as st
    from oracle import cd as ocd
    from oracle import deblend as odb
    from oracle import voronoi as ov

    s, sc = stack
    params, status, _, bg0, _ = _host(st.initial_fits(s, sc))
    names = np.array(_lib.STATUS_NAMES)
    report = []
    for i in range(sc.images):
        img = s[i].cpu().numpy().astype(np.float64)
        sl = sc.image_of(i)
        rows = sc.cells.rows[sl] - [0, i * 768, 0, 0, 0, 0]
        labels = ov.voronoi_labels(rows[:, 4:6], img.shape)
        masks, origins = ocd.cell_stack(labels, rows, 3, img.shape)
        pick = np.linspace(0, len(rows) - 1, 16).astype(int)
        m, o = masks[pick], origins[pick]
        raw = odb.windows(img, o, m.shape[1:])
        border = m & ~binary_erosion(m, structure=np.ones((1, 3, 3)), border_value=0)
        b0 = np.array([np.percentile(r[b], 10) if b.any() else 0.0 for r, b in zip(raw, border)])
        data = np.where(m, raw - b0[:, None, None], 0.0)
        p, st_ = odb.fit_batch(data, m, odb.initial_params(data, m, rows[pick, 4:6] - o), 30)
        gp, gs = params[sl][pick], names[status[sl][pick]]
        np.testing.assert_array_equal(bg0[sl][pick], b0)
        assert np.array_equal(gs, st_)
        both = (gs == "ok")
        err = np.abs(gp[both, 1:3] - p[both, 1:3]).max(initial=0.0)
        report.append((i, len(rows), err))
        assert err <= 1e-6, (i, err)
    print("per-image max centre error vs the FP64 oracle (px):", report)
