"""The Fourier-waist API (the reference's named buffer between the longitude
FFT and the Legendre contraction) against the oracle and against the
engine's own one-call transforms."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("T", [9, 21])
@pytest.mark.parametrize("precision", ["float64", "float32", "split16"])
def test_waist_round_trips(T, precision):
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    t = SphericalHarmonicTransform.create(T, precision=precision)
    ora = DenseSHT(T)
    np_ = t.backend.to_numpy
    tol = 1e-12 if precision == "float64" else 2e-6
    coeff = red_spectrum(T, 3)
    field = ora.inverse(coeff)
    # grid -> waist is the zonal spectrum / nlon cut at m = T.
    w = t.fourier_waist(field)
    assert w.shape == (3, t.grid.nlat, T + 1) and w.bands == 1
    assert rel_max(np_(w.values), ora.fourier(field)) < tol
    # waist -> coefficients is the forward transform.
    c = np_(t.contract_waist(w))
    assert rel_max(c, ora.forward(field)) < tol
    with pytest.raises(RuntimeError, match="consumed"):
        w.values
    # coefficients -> waist -> grid is the inverse transform.
    g = np_(t.waist_to_grid(t.contract_to_waist(coeff)))
    assert rel_max(g, field) < tol
    # the d/dphi table gives the meridional derivative.
    d = np_(t.waist_to_grid(t.contract_to_waist(coeff, t._derivative_basis)))
    assert rel_max(d, ora.inverse_meridional_derivative(coeff)) < tol
    t.check_device()


@pytest.mark.parametrize("precision", ["float64", "split16"])
def test_band_fill_and_drain_match_whole_field(precision):
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    T = 21
    t = SphericalHarmonicTransform.create(T, precision=precision, latitude_bands=3)
    np_ = t.backend.to_numpy
    coeff = red_spectrum(T, 2)
    field = np_(t.inverse(coeff))
    whole = np_(t.contract_waist(t.fourier_waist(field)))
    w = t.open_waist((2,))
    assert w.bands == 3
    for r0, r1 in reversed(w.edges):  # any fill order
        w.fill_band(r0, r1, field[:, r0:r1, :])
    assert np.array_equal(np_(t.contract_waist(w)), whole)
    # gradient, a band at a time, against the one-call gradient
    east, north = (np_(x) for x in t.gradient(coeff))
    waists = t.gradient_waists(coeff)
    for r0, r1 in waists[0].edges:
        e, n = (np_(x) for x in t.gradient_band(waists, r0, r1))
        tol = 1e-12 if precision == "float64" else 2e-6
        assert rel_max(e, east[:, r0:r1]) < tol * 10 and rel_max(n, north[:, r0:r1]) < tol * 10
    t.check_device()


def test_band_fill_errors():
    from b200sht import SphericalHarmonicTransform

    t = SphericalHarmonicTransform.create(9, precision="float64", latitude_bands=2)
    nlat, nlon = t.grid.shape
    w = t.open_waist(())
    w.fill_band(0, 5, np.zeros((5, nlon)))
    with pytest.raises(ValueError, match="overlaps"):
        w.fill_band(3, 6, np.zeros((3, nlon)))
    with pytest.raises(ValueError, match="are not the waist's"):
        w.fill_band(5, 7, np.zeros((3, nlon)))
    with pytest.raises(RuntimeError, match="unwritten latitude rows"):
        t.contract_waist(w)
