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


@pytest.mark.parametrize("precision", ["split16", "float32"])
def test_ensemble_configuration_against_oracle(precision):
    """The ensemble configuration's shapes -- 32 members at T126 on 192 x 384
    plus the control at T255 on 384 x 768, one batch -- with two planes per
    member (64 at T126) and two at T255: sampled planes of every plan
    against the CPU oracle within 2e-6."""
    import torch

    from b200sht import SphericalHarmonicTransform, TransformBatch
    from b200sht.synthetic import CONTROL_SEED, ensemble_member, red_spectrum
    from oracle.dense_sht import DenseSHT

    members, per = 32, 2
    specs = [(126, 192, 384), (255, 384, 768)]
    plans = [SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, precision=precision)
             for T, nl, no in specs]
    c126 = np.concatenate([ensemble_member(red_spectrum(126, per, CONTROL_SEED), k)
                           for k in range(members)])
    c255 = red_spectrum(255, per, CONTROL_SEED)
    batch = TransformBatch(plans, [members * per, per])
    np_ = plans[0].backend.to_numpy
    grids = batch.inverse([c126, c255])
    coeffs = batch.forward([g.contiguous() for g in grids])
    for (T, nl, no), c, g, f, sample in ((specs[0], c126, grids[0], coeffs[0], [0, 37, 63]),
                                         (specs[1], c255, grids[1], coeffs[1], [0, 1])):
        ora = DenseSHT(T, nlat=nl, nlon=no)
        want_g = ora.inverse(c[sample])
        got_g = np_(g)[sample]
        assert np.max(np.abs(got_g - want_g)) / np.max(np.abs(want_g)) < 2e-6, (T, "inverse")
        want_c = ora.forward(got_g.astype(np.float64))
        got_c = np_(f)[sample]
        w = np.where(np.arange(T + 1) == 0, 1.0, 2.0)
        rel = np.sqrt(np.sum(w * np.abs(got_c - want_c) ** 2) / np.sum(w * np.abs(want_c) ** 2))
        assert rel < 2e-6, (T, "forward", rel)
    for p in plans:
        p.check_device()
    torch.cuda.synchronize()
