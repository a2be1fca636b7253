"""Voronoi labels on the GPU: bit-exact against the reference's CPU labels (golden) and the oracle."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import voronoi as ov

pytestmark = pytest.mark.gpu


def test_voronoi_matches_reference_golden():
    from imageprocessor_new_b200 import compute_voronoi_labels

    z = np.load(GOLDEN / "voronoi.npz")
    for name in z["names"]:
        seeds, shape = z[f"{name}_seeds"], tuple(z[f"{name}_shape"])
        np.testing.assert_array_equal(compute_voronoi_labels(seeds, shape), z[f"{name}_labels"], err_msg=str(name))


@pytest.mark.parametrize("n, shape", [(0, (20, 30)), (1, (20, 30)), (2, (64, 64)), (3000, (513, 777)),
                                      (20000, (1024, 1024))])
def test_voronoi_random_against_oracle(n, shape):
    from imageprocessor_new_b200 import compute_voronoi_labels

    rng = np.random.default_rng(n)
    seeds = rng.uniform(0, [shape[1], shape[0]], (n, 2))
    np.testing.assert_array_equal(compute_voronoi_labels(seeds, shape), ov.voronoi_labels(seeds, shape))


def test_voronoi_exact_ties_lowest_index():
    from imageprocessor_new_b200 import compute_voronoi_labels

    # Seeds on half-integer lattices: many pixels equidistant from two or four seeds.
    g = np.stack(np.meshgrid(np.arange(0.5, 200, 4.0), np.arange(0.5, 150, 4.0)), -1).reshape(-1, 2)
    rng = np.random.default_rng(1)
    seeds = g[rng.permutation(len(g))]
    np.testing.assert_array_equal(compute_voronoi_labels(seeds, (150, 200)), ov.voronoi_labels(seeds, (150, 200)))
