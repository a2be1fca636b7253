"""The multi-GPU sharding of tiled detection (imageprocessor_new_b200.shard), run as gloo ranks on
the CPU with the oracle doing each rank's band work: the sharded result must equal the single-process
oracle of the same tiled rules (global Otsu from summed row-shard histograms, round-robin bands,
gather in band order, dedupe)."""

import os
import socket

import numpy as np
import pytest
import torch

from imageprocessor_new_b200 import shard
from oracle import centers as oc
from oracle import segment as osg

KW = dict(threshold="otsu", invert=False, area_min=1, area_max=400, pad=3, refine_method="weighted",
          connectivity=8, small_feature_max=12.0)


class OracleBandOps:
    device = "cpu"

    def histogram(self, rows, step):
        sub = np.ascontiguousarray(rows[::step, ::step])
        hist = np.bincount(sub.ravel(), minlength=shard.NBINS).astype(np.int64)
        return torch.from_numpy(hist), torch.tensor([int(sub.min()), int(sub.max())], dtype=torch.int64), sub.size

    def otsu(self, hist, value_range, total, dtype):
        h = hist.numpy()
        return osg.otsu_from_histogram(h[:256] if np.dtype(dtype) == np.uint8 else h, total)

    def detect(self, band, fixed_threshold):
        kw = dict(KW)
        c = oc.detect_centers(band, fixed_threshold=fixed_threshold, **kw)
        return c[np.isfinite(c).all(axis=1)]

    def dedupe(self, points, eps):
        return oc.dedupe(points, eps)


def _page():
    from imageprocessor_new_b200 import synthetic

    return np.ascontiguousarray(synthetic.page_square(1).image[:520, :400])


def _worker(rank, world, port, tile_h, overlap, mode, out_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        got = shard.detect_tiled_sharded(_page(), tile_h=tile_h, overlap=overlap, threshold_mode=mode,
                                         ops=OracleBandOps())
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), got)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,tile_h,overlap,mode", [(2, 160, 32, "auto"), (3, 128, 40, "global"),
                                                       (2, 200, 64, "per_tile")])
def test_sharded_tiled_detection_equals_single_process(tmp_path, world, tile_h, overlap, mode):
    import torch.multiprocessing as mp

    mp.spawn(_worker, args=(world, _free_port(), tile_h, overlap, mode, str(tmp_path)), nprocs=world, join=True)
    want = oc.detect_tiled(_page(), tile_h=tile_h, overlap=overlap, threshold_mode=mode, **KW)
    for rank in range(world):
        got = np.load(tmp_path / f"rank{rank}.npy")
        assert got.shape == want.shape
        np.testing.assert_array_equal(got, want)


def test_plans_cover_every_row_and_unit_once():
    bands = shard.band_plan(1000, 300, 64)
    keep = np.concatenate([np.arange(b.keep_lo, b.keep_hi) for b in bands])
    np.testing.assert_array_equal(keep, np.arange(1000))
    for world in (1, 2, 3, 8):
        mine = sorted(b.index for r in range(world) for b in shard.bands_of_rank(bands, r, world))
        assert mine == list(range(len(bands)))
        units = [u for r in range(world) for u in shard.units_of_rank(13, r, world)]
        assert units == list(range(13))
        rows = [shard.sampled_rows_of_rank(1001, 4, r, world) for r in range(world)]
        sampled = np.concatenate([np.arange(r0, r1)[::4] for r0, r1 in rows if r1 > r0])
        np.testing.assert_array_equal(sampled, np.arange(1001)[::4])
    with pytest.raises(ValueError):
        shard.band_plan(100, 50, 50)


def _cd_pages():
    from imageprocessor_new_b200 import synthetic

    return [synthetic.gaussian_lattice(r, shape=(90, 150), seed=k)[0] for k, r in enumerate((2.0, 2.67, 2.2, 2.5,
                                                                                          3.0))]


def _oracle_summary(page):
    from oracle import cd as ocd

    r = ocd.measure_cds(page, methods=("gaussian", "halfmax"), area_max=400)
    return {"seeds": r["seeds"], "cd": {m: r["measurements"][m]["metrics"]["cd_equivalent_px"]
                                        for m in ("gaussian", "halfmax")}, "passes": r["passes"]}


def _cd_worker(rank, world, port, dst, out_dir):
    import pickle

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        got = shard.measure_cds_sharded(_cd_pages(), measure=_oracle_summary, dst=dst)
        with open(os.path.join(out_dir, f"cd{rank}.pkl"), "wb") as f:
            pickle.dump(got, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dst", [(2, 0), (3, None)])
def test_sharded_measure_cds_gathers_pages_in_order(tmp_path, world, dst):
    """Pages split into contiguous runs per rank, each measured once (the oracle stands in for each
    rank's GPU), results gathered in page order: equal to measuring every page in one process."""
    import pickle

    import torch.multiprocessing as mp

    mp.spawn(_cd_worker, args=(world, _free_port(), dst, str(tmp_path)), nprocs=world, join=True)
    want = [_oracle_summary(p) for p in _cd_pages()]
    for rank in range(world):
        with open(tmp_path / f"cd{rank}.pkl", "rb") as f:
            got = pickle.load(f)
        if dst is not None and rank != dst:
            assert got is None
            continue
        assert len(got) == len(want)
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g["seeds"], w["seeds"])
            assert g["passes"] == w["passes"]
            for m in w["cd"]:
                np.testing.assert_array_equal(g["cd"][m], w["cd"][m])
