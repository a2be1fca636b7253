"""Result files (save_cd_results / load_cd_results) against folders written by the reference's own
save_cd_results (tests/golden/results_full, results_compact; subpx/cd.py:872-1131): the loader reads
them, and the writer produces the same CSV text and NPZ keys from the same result."""

import numpy as np
import pytest

from conftest import GOLDEN

FULL = GOLDEN / "results_full"
COMPACT = GOLDEN / "results_compact"


def _load_full():
    from imageprocessor_new_b200.results import load_cd_results

    return load_cd_results(FULL)


def test_loader_reads_reference_full_folder():
    res = _load_full()
    with np.load(FULL / "raw_data.npz") as z:
        np.testing.assert_array_equal(res.seeds_xy, z["seeds_xy"])
        np.testing.assert_array_equal(res.cell_labels, z["cell_labels"])
        np.testing.assert_array_equal(res.background_map, z["background_map"])
        for m in ("gaussian", "halfmax"):
            got = res.measurements[m]
            np.testing.assert_array_equal(got.contours_xy, z[f"{m}_contours_xy"])
            np.testing.assert_array_equal(got.status, z[f"{m}_status"])
            np.testing.assert_array_equal(got.metrics["cd_equivalent_px"], z[f"{m}_cd_equivalent_px"])
        np.testing.assert_array_equal(res.mean_intensity, z["mean_intensity"])
    assert res.meta["n_angles"] == 128 and res.deblend_model["tile_px"] > 0


def test_writer_reproduces_reference_tables_and_keys(tmp_path):
    from imageprocessor_new_b200.results import save_cd_results

    res = _load_full()
    paths = save_cd_results(res, tmp_path / "full")
    for name in ("measurements.csv", "cells.csv", "contours.csv"):
        assert paths[name].read_text() == (FULL / name).read_text(), name
    with np.load(paths["raw_data.npz"]) as a, np.load(FULL / "raw_data.npz") as b:
        assert sorted(a.files) == sorted(b.files)
        for key in b.files:
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    import json

    ours, ref = (json.loads(p.read_text()) for p in (paths["manifest.json"], FULL / "manifest.json"))
    assert set(ours) == set(ref)
    assert ours["methods"] == ref["methods"] and ours["files"] == ref["files"]


def test_compact_writer_keys_match_reference(tmp_path):
    from imageprocessor_new_b200.results import save_cd_results

    res = _load_full()
    with np.load(COMPACT / "raw_data.npz") as z:  # a full file keeps no geometry: take the measured one
        for m, measured in res.measurements.items():
            prefix = f"{m}_geometry_"
            measured.geometry = {k[len(prefix):]: z[k] for k in z.files if k.startswith(prefix)}
    paths = save_cd_results(res, tmp_path / "compact", compact=True)
    assert "contours.csv" not in paths
    assert paths["measurements.csv"].read_text() == (COMPACT / "measurements.csv").read_text()
    with np.load(paths["raw_data.npz"]) as a, np.load(COMPACT / "raw_data.npz") as b:
        assert sorted(a.files) == sorted(b.files)
        for key in b.files:
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)


def test_summaries_are_rejected(tmp_path):
    from imageprocessor_new_b200.results import save_cd_results
    from imageprocessor_new_b200.types import CDSummary

    with pytest.raises(ValueError, match="summary_only=False"):
        save_cd_results(CDSummary(seeds_xy=np.zeros((0, 2)), measurements={}), tmp_path)
