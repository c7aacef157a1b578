"""Batched plans (one merged Legendre launch per direction) against the same
plans run one by one, and against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(precision):
    from b200sht import SphericalHarmonicTransform

    a = SphericalHarmonicTransform.create(21, precision=precision)
    b = SphericalHarmonicTransform.create(62, nlat=94, nlon=192, dealias_factor=1.49,
                                          precision=precision)
    return a, b


@pytest.mark.parametrize("precision", ["float64", "float32", "split16"])
def test_batch_equals_single_plan_calls(precision):
    from b200sht import TransformBatch
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    a, b = _pair(precision)
    ca, cb = red_spectrum(21, 3), red_spectrum(62, 5, seed=7)
    batch = TransformBatch([a, b], [3, 5])
    np_ = a.backend.to_numpy
    ga, gb = (np_(x) for x in batch.inverse([ca, cb]))
    fa, fb = (np_(x) for x in batch.forward([ga, gb]))
    # Every tile of the merged launch computes exactly what it computes in a
    # single-plan launch.
    assert np.array_equal(ga, np_(a.inverse(ca)))
    assert np.array_equal(gb, np_(b.inverse(cb)))
    assert np.array_equal(fa, np_(a.forward(ga)))
    assert np.array_equal(fb, np_(b.forward(gb)))
    tol = 1e-12 if precision == "float64" else 2e-6
    for t, c, g, f, df in ((a, ca, ga, fa, 1.5), (b, cb, gb, fb, 1.49)):
        ora = DenseSHT(t.truncation, nlat=t.grid.nlat, nlon=t.grid.nlon, dealias_factor=df)
        want = ora.inverse(c)
        assert np.max(np.abs(g - want)) / np.max(np.abs(want)) < tol
        back = ora.forward(g.astype(np.float64))
        assert np.max(np.abs(f - back)) / np.max(np.abs(back)) < tol
    a.check_device()
    b.check_device()


def test_batch_argument_errors():
    from b200sht import SphericalHarmonicTransform, TransformBatch

    a, b = _pair("float32")
    s = SphericalHarmonicTransform.create(21, precision="split16")
    with pytest.raises(ValueError, match="twice"):
        TransformBatch([a, a], [1, 1])
    with pytest.raises(ValueError, match="precision"):
        TransformBatch([a, s], [1, 1])
    with pytest.raises(ValueError, match="1 to 4"):
        TransformBatch([], [])
    batch = TransformBatch([a, b], [2, 2])
    with pytest.raises(ValueError, match="does not hold"):
        batch.inverse([np.zeros((3, 22, 22), complex), np.zeros((2, 63, 63), complex)])
