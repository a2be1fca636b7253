"""CUDA segmentation (Otsu, triangle, CCL + stats) against the golden fixtures and the oracle."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import segment as osg

pytestmark = pytest.mark.gpu


def _load(name):
    return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)


def test_otsu_and_triangle_bit_exact():
    from imageprocessor_new_b200 import _device as dev, segment

    z = _load("thresholds")
    for i in range(int(z["n"])):
        img = z[f"img{i}"]
        t = segment.otsu(dev.upload(img)).item()
        assert t == z["otsu"][i], (i, t, z["otsu"][i])
        if img.dtype == np.uint8:
            assert segment.triangle(dev.upload(img)).item() == z["triangle"][i]


def test_otsu_strided_and_page():
    from imageprocessor_new_b200 import _device as dev, segment, synthetic

    page = synthetic.page_square(0).image
    for step in (1, 2, 4):
        got = segment.otsu(dev.upload(page), step=step).item()
        assert got == osg.otsu_threshold(np.ascontiguousarray(page[::step, ::step]))


@pytest.mark.parametrize("conn", [8, 4])
def test_ccl_matches_opencv_golden(conn):
    from imageprocessor_new_b200 import segment

    z = _load("ccl")
    for i in range(int(z["n"])):
        shape = tuple(z[f"shape{i}"])
        mask = np.unpackbits(z[f"mask{i}"])[: shape[0] * shape[1]].reshape(shape).astype(np.uint8) * 255
        res = segment.connected_components_stats(mask, connectivity=conn)
        np.testing.assert_array_equal(res.labels, z[f"labels{i}_{conn}"], err_msg=f"case {i}")
        np.testing.assert_array_equal(res.stats, z[f"stats{i}_{conn}"], err_msg=f"case {i}")
        np.testing.assert_array_equal(res.centroids[1:], z[f"cent{i}_{conn}"][1:], err_msg=f"case {i}")
        assert res.num_labels == len(z[f"stats{i}_{conn}"])


@pytest.mark.parametrize("shape", [(1, 1), (1, 97), (97, 1), (33, 65), (64, 128), (257, 511), (1024, 1024)])
@pytest.mark.parametrize("conn", [8, 4])
def test_ccl_random_sizes_against_oracle(shape, conn):
    from imageprocessor_new_b200 import segment

    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    for p in (0.0, 0.3, 0.6, 1.0):
        fg = rng.random(shape) < p
        res = segment.connected_components_stats(fg.astype(np.uint8), connectivity=conn)
        num, labels, stats, cents = osg.label_components(fg, conn)
        assert res.num_labels == num
        np.testing.assert_array_equal(res.labels, labels)
        np.testing.assert_array_equal(res.stats[1:], stats[1:])
        np.testing.assert_array_equal(res.centroids[1:], cents[1:])


def test_ccl_spirals_cross_many_tiles():
    """Long components that wind through many 32x64 tiles and meet across tile borders."""
    from imageprocessor_new_b200 import segment

    h, w = 300, 400
    fg = np.zeros((h, w), bool)
    fg[::4, :] = True
    fg[:, ::97] = True
    fg[150, :] = False
    fg[np.arange(h), (np.arange(h) * 7) % w] = True
    for conn in (8, 4):
        res = segment.connected_components_stats(fg.astype(np.uint8), connectivity=conn)
        num, labels, stats, cents = osg.label_components(fg, conn)
        assert res.num_labels == num
        np.testing.assert_array_equal(res.labels, labels)
        np.testing.assert_array_equal(res.stats[1:], stats[1:])


def test_ccl_deterministic():
    from imageprocessor_new_b200 import segment

    rng = np.random.default_rng(0)
    fg = (rng.random((512, 700)) < 0.5).astype(np.uint8)
    a = segment.connected_components_stats(fg)
    b = segment.connected_components_stats(fg)
    np.testing.assert_array_equal(a.labels, b.labels)
    np.testing.assert_array_equal(a.stats, b.stats)


def test_large_uploads_round_trip():
    """Large host arrays go up in overlapped chunks (ragged last chunk, odd dtypes): every byte
    arrives, and several uploads in flight at once keep their own pinned blocks."""
    from imageprocessor_new_b200 import _device as dev

    rng = np.random.default_rng(5)
    arrays = [rng.integers(0, 65536, (4099, 4111), dtype=np.uint16),
              rng.random((1031, 4097)),
              rng.integers(0, 255, (70003, 1029), dtype=np.uint8)[::2]]  # non-contiguous
    ups = [dev.upload(a) for a in arrays]
    for a, d in zip(arrays, ups):
        np.testing.assert_array_equal(d.cpu().numpy(), a)
