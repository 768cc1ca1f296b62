"""The ellipse / ellipsoid generator (notebooks/gen_ellipsoid.py:12-38)
against a cell-by-cell restatement, on the parameter sets of the
reference's own test (gen_ellipsoid.py:67-76)."""
import itertools

import numpy as np
import pytest

from janus_b200.microstructures import ellipsoid

CASES = [((0.3, 0.4), (1.0, 1.0), (100, 100)),
         ((0.3, 0.4), (0.8, 1.0), (80, 100)),
         ((0.3, 0.4), (0.6, 0.8), (60, 80)),
         ((0.3, 0.4), (0.4, 0.6), (40, 60)),
         ((0.3, 0.4), (0.4, 0.6), (50, 50)),
         ((0.3, 0.4, 0.5), (1.0, 1.0, 1.0), (40, 40, 40)),
         ((0.3, 0.4, 0.5), (0.8, 1.0, 1.2), (32, 40, 48)),
         ((0.3, 0.4, 0.5), (0.4, 0.6, 0.8), (20, 30, 40)),
         ((0.3, 0.4, 0.5), (0.4, 0.6, 0.8), (25, 25, 25))]


def _cells(radii, size, shape):
    out = np.zeros(shape, dtype=np.int8)
    axes = [np.linspace(-0.5 * L * (n - 1) / n, 0.5 * L * (n - 1) / n, num=n)
            for L, n in zip(size, shape)]
    for idx in itertools.product(*[range(n) for n in shape]):
        s = sum((axes[d][i] / radii[d]) ** 2 for d, i in enumerate(idx))
        out[idx] = 1 if s <= 1 else 0
    return out


@pytest.mark.parametrize("radii, size, shape", CASES)
def test_ellipsoid_cells(radii, size, shape):
    got = ellipsoid(radii, size, shape)
    assert got.dtype == np.int8 and got.shape == shape
    np.testing.assert_array_equal(got, _cells(radii, size, shape))


def test_ellipsoid_rejects_mixed_lengths():
    with pytest.raises(ValueError):
        ellipsoid((0.3, 0.4), (1.0, 1.0, 1.0), (10, 10))
