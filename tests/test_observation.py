"""Agent observation sphere (Agent.h:147-192) from the library, against the formula restated
here in float32: a spiral of n unit directions, latitude parameter s over (-1, 1)."""
import math

import numpy as np
import pytest

from nanomap_b200 import api as A
from nanomap_b200._native import NanomapError


def _sphere(n):
    x = np.float32(0.1 + 1.2 * n)
    start = np.float32(-1.0 + 1.0 / (n - 1.0))
    inc = np.float32((2.0 - 2.0 / (n - 1.0)) / (n - 1.0))
    out = np.zeros((n, 3), np.float32)
    for i in range(n):
        s = np.float32(start + np.float32(i) * inc)
        lon = np.float32(s * x)
        lat = np.float32((math.pi / 2.0) * math.copysign(1.0, float(s)) * (1.0 - math.sqrt(1.0 - abs(float(s)))))
        p = np.array([np.cos(lon) * np.cos(lat), np.sin(lon) * np.cos(lat), np.sin(lat)], np.float32)
        out[i] = p / np.float32(np.sqrt((p * p).sum()))
    return out


@pytest.mark.parametrize("n", [2, 3, 32, 500])
def test_observation_sphere_matches_formula(n):
    got = A.observation_sphere(n)
    assert got.shape == (n, 3)
    np.testing.assert_allclose(got, _sphere(n), atol=2e-6)
    np.testing.assert_allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-6)
    if n >= 32:  # spread over both hemispheres
        assert got[:, 2].min() < -0.9 and got[:, 2].max() > 0.9


def test_observation_sphere_rejects_fewer_than_two():
    with pytest.raises(NanomapError):
        A.observation_sphere(1)
