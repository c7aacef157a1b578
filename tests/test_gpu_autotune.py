"""The autotuner's settings: every combination it may pick computes the same
transform within the precision's bar, and it keeps the fastest."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    w = np.where(np.arange(a.shape[-1]) == 0, 1.0, 2.0)[None, :]
    return float(np.sqrt(np.sum(w * np.abs(a - b) ** 2) / np.sum(w * np.abs(b) ** 2)))


def test_every_setting_meets_the_bar_and_tune_keeps_the_fastest(tmp_path):
    from b200sht import SphericalHarmonicTransform
    from b200sht.autotune import _candidates, get_tuning, set_tuning, tune
    from b200sht.synthetic import red_spectrum

    kw = dict(nlat=94, nlon=192, dealias_factor=1.49)
    f64 = SphericalHarmonicTransform.create(62, precision="float64", **kw)
    t = SphericalHarmonicTransform.create(62, precision="split16", **kw)
    np_ = t.backend.to_numpy
    coeff = red_spectrum(62, 6)
    grid = f64.inverse(coeff)
    want = np_(f64.forward(grid))
    cands = _candidates(t)
    # {TC x 2 orders, SIMT x 2 tile shapes} x {register FFT, Stockham FFT}
    assert len(cands) == 8
    for cand in cands:
        set_tuning(t, **cand)
        assert get_tuning(t) == cand
        assert rel_l2(np_(t.forward(grid.float())), want) < 2e-6
        assert np.max(np.abs(np_(t.inverse(coeff)) - np_(grid))) / np.max(np.abs(np_(grid))) < 2e-6
    report = tune(t, 6, repeats=2, warmup=1, cache=tmp_path / "tune.json")
    assert report["best"] == get_tuning(t)
    assert report["ms"][min(report["ms"], key=report["ms"].get)] == min(report["ms"].values())
    again = tune(t, 6, cache=tmp_path / "tune.json")
    assert again["cached"] and again["best"] == report["best"]
    t.check_device()


def test_tuning_errors():
    from b200sht import SphericalHarmonicTransform
    from b200sht.autotune import set_tuning

    f64 = SphericalHarmonicTransform.create(21, precision="float64")
    with pytest.raises(ValueError, match="register-resident"):
        set_tuning(f64, fft=0)
    with pytest.raises(ValueError, match="split16"):
        set_tuning(f64, contraction=1)
    with pytest.raises(ValueError, match="unknown tuning setting"):
        set_tuning(f64, band=3)
    with pytest.raises(ValueError, match="SHT_TUNE_ACCUMULATORS"):
        set_tuning(f64, accumulators=3)


@pytest.mark.parametrize("acc", [0, 1, 2])
def test_accumulator_plans_meet_the_bar_at_t255(acc):
    from b200sht import SphericalHarmonicTransform, VorticityDivergenceOperator
    from b200sht.autotune import set_tuning
    from b200sht.synthetic import red_spectrum

    kw = dict(nlat=384, nlon=768)
    f64 = SphericalHarmonicTransform.create(255, precision="float64", **kw)
    t = SphericalHarmonicTransform.create(255, precision="split16", **kw)
    set_tuning(t, accumulators=acc)
    np_ = t.backend.to_numpy
    coeff = red_spectrum(255, 4)
    grid = f64.inverse(coeff)
    assert rel_l2(np_(t.forward(grid.float())), np_(f64.forward(grid))) < 2e-6
    g = np_(t.inverse(coeff))
    assert np.max(np.abs(g - np_(grid))) / np.max(np.abs(np_(grid))) < 2e-6
    u64, v64 = VorticityDivergenceOperator(f64).wind_from_vordiv(coeff, coeff[::-1].copy())
    u, v = VorticityDivergenceOperator(t).wind_from_vordiv(coeff, coeff[::-1].copy())
    assert np.max(np.abs(np_(u) - np_(u64))) / np.max(np.abs(np_(u64))) < 2e-6
    t.check_device()


@pytest.mark.parametrize("precision", ["float32", "split16"])
def test_simt_tile_shapes_agree_bit_for_bit(precision):
    """The two FP32 SIMT tile shapes run every output's FFMA chain in the same
    order, so they return the same bits (on a split16 plan through the SIMT
    contraction switch)."""
    import torch

    from b200sht import SphericalHarmonicTransform
    from b200sht.autotune import set_tuning
    from b200sht.synthetic import red_spectrum

    t = SphericalHarmonicTransform.create(127, precision=precision)
    if precision == "split16":
        set_tuning(t, contraction=1)
    coeff = red_spectrum(127, 5)
    out = []
    for tile in (0, 1):
        set_tuning(t, simt_tile=tile)
        g = t.inverse(coeff)
        out.append((g.clone(), t.forward(g).clone()))
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    f64 = SphericalHarmonicTransform.create(21, precision="float64")
    with pytest.raises(ValueError, match="FP32 tile shape"):
        set_tuning(f64, simt_tile=1)
    t.check_device()
