"""The unmeasured-tile interpolation of the background map (cached barycentric weights) against the
reference's LinearNDInterpolator + nearest-tile rule, bit for bit (no GPU needed)."""

import numpy as np
import pytest


def _reference(free_med, measured, tile, shape):
    from scipy.interpolate import LinearNDInterpolator
    from scipy.spatial import Delaunay, cKDTree

    from imageprocessor_new_b200.deblend import tile_centers

    yc, xc = tile_centers(tile, shape)
    grid = np.stack(np.meshgrid(yc, xc, indexing="ij"), axis=-1)
    known, values = grid[measured], free_med[measured]
    try:
        tri = Delaunay(known) if len(values) >= 3 else None
    except Exception:
        tri = None
    medians = free_med.copy()
    missing = ~measured
    medians[missing] = np.nan
    if tri is not None:
        medians[missing] = LinearNDInterpolator(tri, values)(grid[missing])
    still = missing & np.isnan(medians)
    medians[still] = values[cKDTree(known).query(grid[still])[1]]
    return medians


@pytest.mark.parametrize("shape, tile, frac", [((8192, 8192), 96, 0.05), ((1024, 1024), 128, 0.5),
                                                ((300, 500), 64, 0.3), ((256, 256), 128, 0.75),
                                                ((200, 700), 100, 0.0)])
def test_interpolate_tiles_matches_linearnd(shape, tile, frac):
    from imageprocessor_new_b200.deblend import interpolate_tiles

    rng = np.random.default_rng(7)
    ny, nx = -(-shape[0] // tile), -(-shape[1] // tile)
    for _ in range(4):
        measured = rng.random((ny, nx)) >= frac
        measured.flat[rng.integers(0, measured.size)] = False
        if not measured.any():
            measured.flat[0] = True
        free_med = rng.normal(1000.0, 5.0, (ny, nx))
        # twice with the same mask (the second call uses the cached weights), new values each time
        for _ in range(2):
            free_med = free_med + rng.normal(0.0, 1.0, (ny, nx))
            np.testing.assert_array_equal(interpolate_tiles(free_med, measured, tile, shape),
                                          _reference(free_med, measured, tile, shape))
