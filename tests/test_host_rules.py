"""Host-side rules of the CD driver that need no GPU: the median foot_area_ratio's threshold takes
(NumPy's nanmedian rule, computed on torch tensors) and the tail family's default pitch."""

import numpy as np
import pytest
import torch


@pytest.mark.parametrize("n", [1, 2, 7, 64, 65])
def test_device_nanmedian_is_numpys(n):
    from imageprocessor_new_b200.cd import _nanmedian_device

    rng = np.random.default_rng(n)
    v = rng.normal(size=n)
    v[rng.random(n) < 0.2] = np.nan
    got = _nanmedian_device(torch.from_numpy(v))
    want = np.nanmedian(v) if np.isfinite(v).any() else np.nan
    if np.isnan(want):
        assert np.isnan(got)
    else:
        assert got == want  # the mean of the two middle values for an even count, bit for bit


def test_device_nanmedian_empty():
    from imageprocessor_new_b200.cd import _nanmedian_device

    assert np.isnan(_nanmedian_device(torch.tensor([np.nan, np.nan], dtype=torch.float64)))
    assert np.isnan(_nanmedian_device(torch.zeros(0, dtype=torch.float64)))


def test_median_pitch_needs_two_holes():
    """measure_invariant's default pitch (median nearest-neighbour distance of the fitted centres):
    none for fewer than two finite centres (the windows then use the stack's larger side)."""
    from oracle.invariant import median_pitch

    class State:
        params = np.array([[1.0, 3.0, 4.0, 0, 0, 0], [1.0, np.nan, 2.0, 0, 0, 0]])

    assert median_pitch(State, np.zeros((2, 2))) is None
    State.params = np.array([[1.0, 0.0, 0.0, 0, 0, 0], [1.0, 3.0, 4.0, 0, 0, 0], [1.0, 9.0, 4.0, 0, 0, 0]])
    assert median_pitch(State, np.zeros((3, 2))) == 5.0
