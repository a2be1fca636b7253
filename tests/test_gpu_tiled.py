"""detect_centers(tile_h=...) on the GPU against the reference's tiled rules (golden) and dedupe."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import centers as oc

pytestmark = pytest.mark.gpu


def _sorted(a):
    return a[np.lexsort((a[:, 1], a[:, 0]))]


def test_tiled_matches_reference_rules():
    from imageprocessor_new_b200 import detect_centers_tiled

    z = np.load(GOLDEN / "tiled.npz")
    with pytest.warns(DeprecationWarning):
        res = detect_centers_tiled(z["img"], tile_h=int(z["tile_h"]), overlap=int(z["overlap"]), backend="gpu",
                                   threshold="otsu", area_max=200, refine="logquad")
    want = z["centers"]
    assert res.centers_xy.shape == want.shape
    np.testing.assert_allclose(_sorted(res.centers_xy), _sorted(want), rtol=0, atol=1e-9)


@pytest.mark.parametrize("n, eps", [(0, 1.5), (1, 1.5), (500, 1.5), (20000, 1.5), (3000, 0.0), (4000, 6.0)])
def test_dedupe_matches_oracle(n, eps):
    from imageprocessor_new_b200.tiled import dedupe_centers

    rng = np.random.default_rng(n)
    base = rng.uniform(0, 2000, (n, 2))
    # Near duplicates, exact duplicates and chains.
    dup = base[: n // 3] + rng.normal(0, 0.5, (n // 3, 2))
    pts = np.concatenate([base, dup, base[: n // 10]]) if n else np.zeros((0, 2))
    pts = pts[rng.permutation(len(pts))]
    got = dedupe_centers(pts, eps=eps)
    want = oc.dedupe(pts, eps)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)


def test_tiled_per_tile_threshold_and_bad_overlap():
    from imageprocessor_new_b200 import detect_centers, synthetic

    page = synthetic.page_square(2).image
    res = detect_centers(page, backend="gpu", tile_h=300, overlap=40, threshold="otsu", threshold_mode="per_tile",
                         area_max=400, refine="weighted")
    full = detect_centers(page, backend="gpu", threshold="otsu", area_max=400, refine="weighted").centers_xy
    # Bands of 300 rows see whole holes (pitch 32) in their keep zones: the same centres.
    assert abs(len(res.centers_xy) - len(full)) <= 2
    with pytest.raises(ValueError):
        detect_centers(page, backend="gpu", tile_h=100, overlap=100)


def test_histogram_shards_give_the_global_otsu():
    import torch

    from imageprocessor_new_b200 import segment, shard, synthetic

    page = synthetic.page_staggered(2, shape=(1500, 1300)).image
    ops = shard.GpuBandOps()
    ds = 4
    hist = torch.zeros(shard.NBINS, dtype=torch.int64, device="cuda")
    lo, hi, total = None, None, 0
    for rank in range(3):
        r0, r1 = shard.sampled_rows_of_rank(page.shape[0], ds, rank, 3)
        h, rng, n = ops.histogram(page[r0:r1], ds)
        hist += h
        lo = int(rng[0]) if lo is None else min(lo, int(rng[0]))
        hi = int(rng[1]) if hi is None else max(hi, int(rng[1]))
        total += n
    got = ops.otsu(hist, torch.tensor([lo, hi], dtype=torch.int64, device="cuda"), total, page.dtype)
    want = float(segment.otsu(torch.from_numpy(page).cuda(), step=ds).item())
    assert got == want


def test_sharded_tiled_detection_on_one_rank_matches_detect_centers():
    import os
    import socket

    import torch.distributed as dist

    from imageprocessor_new_b200 import detect_centers, shard, synthetic

    page = synthetic.page_square(5).image
    kw = dict(threshold="otsu", invert=False, area_min=1, area_max=400, pad=3, refine="logquad", connectivity=8,
              small_feature_max=12.0)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        got = shard.detect_tiled_sharded(page, tile_h=300, overlap=64, ops=shard.GpuBandOps(**kw))
    finally:
        dist.destroy_process_group()
    want = detect_centers(page, backend="gpu", tile_h=300, overlap=64, **kw).centers_xy
    np.testing.assert_array_equal(got, want)


def _tiled_kwargs():
    return dict(threshold="otsu", invert=False, area_min=1, area_max=400, pad=3, refine="logquad", connectivity=8,
                small_feature_max=12.0, tile_h=1024, overlap=128, threshold_mode="global", otsu_downsample=4,
                thr_scale=0.8, dedupe_eps=1.5, device=0)


@pytest.mark.parametrize("morph", [(0, 0), (1, 1)])
def test_band_graphs_match_the_eager_bands(morph):
    """The graph-captured band pipeline gives the eager path's centres bit for bit (bands of two
    heights, so two graphs), also with opening / closing, and again on a second replay."""
    from imageprocessor_new_b200 import synthetic, tiled

    page = synthetic.page_staggered(3, shape=(2900, 1536)).image
    kw = dict(_tiled_kwargs(), morph_open=morph[0], morph_close=morph[1])
    eager = tiled.detect_tiled(page, use_graphs=False, **kw)
    graphs = tiled.detect_tiled(page, use_graphs=True, **kw)
    assert graphs.meta["band_graphs"] and not eager.meta["band_graphs"]
    assert len(eager.centers_xy) > 1000
    np.testing.assert_array_equal(graphs.centers_xy, eager.centers_xy)
    np.testing.assert_array_equal(tiled.detect_tiled(page, use_graphs=True, **kw).centers_xy, eager.centers_xy)


def test_band_graph_overflow_takes_the_eager_path(monkeypatch):
    """A band with more components than the captured capacity sends the page down the eager path."""
    from imageprocessor_new_b200 import synthetic, tiled

    page = synthetic.page_staggered(4, shape=(1500, 1024)).image
    eager = tiled.detect_tiled(page, use_graphs=False, **_tiled_kwargs())
    assert len(eager.centers_xy) > 2 * 1024
    monkeypatch.setattr(tiled, "BAND_PX_PER_COMPONENT", 1 << 30)  # capacity 1024 < components per band
    res = tiled.detect_tiled(page, use_graphs=True, **_tiled_kwargs())
    assert tiled.band_capacity(1024, 1024, 5000) == 1024
    assert not res.meta["band_graphs"]
    np.testing.assert_array_equal(res.centers_xy, eager.centers_xy)
