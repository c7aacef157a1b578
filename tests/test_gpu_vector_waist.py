"""The vector analysis through the Fourier waist, and the contraction seam.

* ``_wind_fourier``, ``vordiv_from_wind_waist``, ``_vordiv_from_fourier``
  (on a waist and on a raw full-width zonal spectrum) and
  ``divergence_from_fourier`` against the reference's own outputs
  (tests/golden/make_golden_vector.py), at the parity bars of the other
  transform tests: FP64 within 1e-12 of the largest output, FP32 and split
  within 2e-6 relative spectral L2.
* A waist filled by latitude bands gives the resident waist's result bit
  for bit.
* The census: replacing ``SphericalHarmonicTransform._batched_contract`` the
  way the reference's census tool does
  (tools/arwen_global_transform_census.py:64-140) records the same calls,
  tables and plane counts as the reference's transform (census.json).
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

CASES = ["vector_waist_t21.npz", "vector_waist_t62.npz"]
PRECISIONS = ["float64", "float32", "split16"]


def _make(g, precision):
    from b200sht import SphericalHarmonicTransform

    return SphericalHarmonicTransform.create(
        int(g["truncation"]), nlat=int(g["nlat"]), nlon=int(g["nlon"]),
        dealias_factor=float(g["dealias_factor"]), precision=precision)


def _rel_l2(a, b):
    w = np.where(np.arange(a.shape[-1]) == 0, 1.0, 2.0)
    return float(np.sqrt(np.sum(w * np.abs(a - b) ** 2) / np.sum(w * np.abs(b) ** 2)))


def _rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _check(got, want, precision):
    if precision == "float64":
        assert _rel_max(got, want) < 1e-12
    else:
        assert _rel_l2(got, want) < 2e-6


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("case", CASES)
def test_vector_waist_halves_match_reference(case, precision):
    from b200sht import VorticityDivergenceOperator, build

    build.build()
    g = load_golden(case)
    sht = _make(g, precision)
    vec = VorticityDivergenceOperator(sht)
    np_ = sht.backend.to_numpy
    pair = np.stack([g["u"], g["v"]])
    waist = vec._wind_fourier(pair)
    got = np_(waist.values)
    if precision == "float64":
        assert _rel_max(got, g["waist"]) < 1e-13
    else:
        assert _rel_max(got, g["waist"]) < 2e-6
    z, d = vec.vordiv_from_wind_waist(waist)
    _check(np_(z), g["zeta_waist"], precision)
    _check(np_(d), g["div_waist"], precision)
    raw = np.fft.rfft(pair, axis=-1) / int(g["nlon"])
    z, d = vec._vordiv_from_fourier(raw)
    _check(np_(z), g["zeta_raw"], precision)
    _check(np_(d), g["div_raw"], precision)
    d_only = np_(vec.divergence_from_fourier(vec._wind_fourier(pair)))
    _check(d_only, g["div_only"], precision)
    assert np.all(d_only[..., :, 0].imag == 0)
    sht.check_device()


@pytest.mark.parametrize("precision", ["float64", "split16"])
def test_banded_vector_waist_equals_whole_call(precision):
    import torch

    from b200sht import VorticityDivergenceOperator

    g = load_golden("vector_waist_t62.npz")
    sht = _make(g, precision)
    vec = VorticityDivergenceOperator(sht)
    pair = torch.as_tensor(np.stack([g["u"], g["v"]])).to(sht.backend.device,
                                                          sht.backend.float_dtype)
    # The reference's bit-identity claim: a band-filled waist contracts to
    # the resident waist's coefficients (the direct vordiv_from_wind call
    # skips the waist layout and rounds differently).
    whole = vec.vordiv_from_wind_waist(sht.fourier_waist(pair))
    waist = sht.open_waist(tuple(pair.shape[:-2]), bands=3)
    for r0, r1 in waist.edges:
        waist.fill_band(r0, r1, pair[..., r0:r1, :])
    banded = vec.vordiv_from_wind_waist(waist)
    for a, b in zip(banded, whole):
        assert torch.equal(a, b)
    d = vec.divergence_from_fourier(vec._wind_fourier(pair))
    d_whole = vec.divergence_from_fourier(sht.fourier_waist(pair))
    assert torch.equal(d, d_whole)


def test_divergence_from_fourier_refuses_unpaired_waist():
    from b200sht import VorticityDivergenceOperator

    g = load_golden("vector_waist_t21.npz")
    sht = _make(g, "float32")
    vec = VorticityDivergenceOperator(sht)
    triple = np.stack([g["u"], g["v"], g["u"]])
    with pytest.raises(ValueError, match="leading length 3"):
        vec.divergence_from_fourier(sht.fourier_waist(triple))


def test_contraction_census_matches_reference(monkeypatch):
    """The reference's census hook, applied to the B200 transform, counts the
    reference's contractions: same calls, tables, transposition and planes."""
    from b200sht import SphericalHarmonicTransform, VorticityDivergenceOperator
    from b200sht.synthetic import red_spectrum

    ref = json.loads((GOLDEN / "census.json").read_text())
    t, lead = int(ref["truncation"]), tuple(ref["lead"])
    sht = SphericalHarmonicTransform.create(t, precision="float32")
    vec = VorticityDivergenceOperator(sht)
    coeff = red_spectrum(t, int(np.prod(lead))).reshape(*lead, t + 1, t + 1)
    grid = np.random.default_rng(11).standard_normal((*lead, *sht.grid.shape))
    records = []
    contract = SphericalHarmonicTransform._batched_contract

    def hook(self, values, table, *, transposed=False, **keywords):
        planes = 1
        for extent in values.shape[:-2]:
            planes *= int(extent)
        records.append([str(table), bool(transposed), planes])
        return contract(self, values, table, transposed=transposed, **keywords)

    monkeypatch.setattr(SphericalHarmonicTransform, "_batched_contract", hook)
    calls = {
        "forward": lambda: sht.forward(grid),
        "inverse": lambda: sht.inverse(coeff),
        "inverse_zonal_derivative": lambda: sht.inverse_zonal_derivative(coeff),
        "inverse_meridional_derivative": lambda: sht.inverse_meridional_derivative(coeff),
        "gradient": lambda: sht.gradient(coeff),
        "contract_waist": lambda: sht.contract_waist(sht.fourier_waist(grid)),
        "contract_to_waist": lambda: sht.contract_to_waist(coeff),
        "gradient_waists": lambda: sht.gradient_waists(coeff),
        "wind_from_vordiv": lambda: vec.wind_from_vordiv(coeff, coeff),
        "vordiv_from_wind": lambda: vec.vordiv_from_wind(grid, grid),
        "vordiv_from_wind_waist": lambda: vec.vordiv_from_wind_waist(
            vec._wind_fourier(np.stack([grid, grid]))),
        "divergence_from_fourier": lambda: vec.divergence_from_fourier(
            vec._wind_fourier(np.stack([grid, grid]))),
    }
    assert set(calls) == set(ref["calls"])
    for name, fn in calls.items():
        records.clear()
        fn()
        assert records == ref["calls"][name], name
    # the seam's own count agrees with the hook
    monkeypatch.undo()
    before = sht.contraction_count
    vec.vordiv_from_wind(grid, grid)
    assert sht.contraction_count - before == 2
