"""The CPU oracle against the reference's recorded outputs and closed forms.

These pins are what lets the CUDA parity tests trust the oracle on a host
where the reference itself is absent.
"""
from __future__ import annotations

import json
import math

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle.dense_sht import DenseSHT, gauss_nodes, legendre_table, solve_shifted

CASES = ["sht_t9.npz", "sht_t21.npz", "sht_t31_wide.npz", "sht_t62.npz"]


def _oracle_for(g):
    return DenseSHT(int(g["truncation"]), nlat=int(g["nlat"]), nlon=int(g["nlon"]),
                    dealias_factor=float(g["dealias_factor"]))


def _close(a, b, tol):
    scale = max(1.0, float(np.max(np.abs(b))))
    assert np.max(np.abs(np.asarray(a) - np.asarray(b))) <= tol * scale


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_outputs(case):
    g = load_golden(case)
    o = _oracle_for(g)
    np.testing.assert_allclose(o.mu, g["mu"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(o.w, g["weights"], rtol=1e-14, atol=0)
    tol = 1e-13
    _close(o.forward(g["grid"]), g["forward"], tol)
    _close(g["forward_frozen"], g["forward"], tol)
    _close(o.inverse(g["coeff"]), g["inverse"], tol)
    _close(o.inverse_zonal_derivative(g["coeff"]), g["zonal"], tol)
    _close(o.inverse_meridional_derivative(g["coeff"]), g["meridional"], tol)
    east, north = o.gradient(g["coeff"])
    _close(east * o.radius_m, g["east"] * o.radius_m, tol)
    _close(north * o.radius_m, g["north"] * o.radius_m, tol)
    _close(o.laplacian(g["coeff"]), g["laplacian"], tol)
    _close(o.inverse_laplacian(g["coeff"]) / o.radius_m ** 2,
           g["inverse_laplacian"] / o.radius_m ** 2, tol)
    np.testing.assert_array_equal(o.project(g["project_in"]), g["project_out"])
    wu, wv = o.wind_from_vordiv(g["coeff"], g["coeff2"])
    _close(wu / o.radius_m, g["wind_u"] / o.radius_m, tol)
    _close(wv / o.radius_m, g["wind_v"] / o.radius_m, tol)
    z, d = o.vordiv_from_wind(g["u"], g["v"])
    _close(z * o.radius_m, g["vort"] * o.radius_m, tol)
    _close(d * o.radius_m, g["div"] * o.radius_m, tol)
    check = o.transform_check(seed=19)
    assert check["roundtrip_relative_linf"] < 5e-13
    assert abs(check["roundtrip_relative_linf"] - float(g["check_roundtrip"])) < 5e-13


def test_oracle_closed_form_harmonics():
    """A real field carrying 2 Re(Y_nm) analyses to exactly one at (n, m)
    (the reference's known-answer test, transform.py's analysis claim)."""
    o = DenseSHT(15)
    lat = np.arcsin(o.mu)[:, None]
    lon = (np.arange(o.nlon) * 2 * np.pi / o.nlon)[None, :]
    s, c = np.sin(lat), np.cos(lat)
    harmonics = {
        (0, 0): np.full((o.nlat, o.nlon), 1 / math.sqrt(4 * math.pi)),
        (1, 0): math.sqrt(3 / (4 * math.pi)) * s + 0 * lon,
        (2, 0): math.sqrt(5 / (16 * math.pi)) * (3 * s ** 2 - 1) + 0 * lon,
        (2, 2): 2 * np.real(math.sqrt(15 / (32 * math.pi)) * c ** 2 * np.exp(2j * lon)),
        (3, 2): 2 * np.real(math.sqrt(105 / (32 * math.pi)) * s * c ** 2 * np.exp(2j * lon)),
    }
    for (n, m), f in harmonics.items():
        coeff = o.forward(f)
        assert abs(coeff[n, m] - 1.0) < 5e-15
        coeff[n, m] = 0
        assert np.max(np.abs(coeff)) < 5e-15


def test_oracle_basis_matches_pinned_ynm():
    data = json.loads((GOLDEN / "ynm_reference.json").read_text())
    tables = [data]
    if "scipy_extra" in data:
        tables.append(data["scipy_extra"])
    for tab in tables:
        lat = np.deg2rad(np.asarray(tab["latitude_deg"]))
        lon = np.deg2rad(np.asarray(tab["longitude_deg"]))
        p = legendre_table(12, np.sin(lat))
        for key, row in tab["values"].items():
            n, m = (int(x) for x in key.split(","))
            ours = p[n, m] * np.exp(1j * m * lon)
            ref = np.asarray(row["real"]) + 1j * np.asarray(row["imag"])
            np.testing.assert_allclose(ours, ref, rtol=2e-14, atol=2e-14)


@pytest.mark.parametrize("case", ["helmholtz_t7_l6.npz", "helmholtz_t21_l40.npz"])
def test_oracle_helmholtz_matches_reference(case):
    g = load_golden(case)
    d, th, lp = solve_shifted(g["divergence"], g["theta"], g["lnps"], g["b_matrix"],
                              g["c_matrix"], g["eigenvalues"], g["eigenvectors"],
                              float(g["tau_s"]) * float(g["weight"]), float(g["radius_m"]))
    for ours, ref in ((d, g["out_divergence"]), (th, g["out_theta"]), (lp, g["out_lnps"])):
        np.testing.assert_allclose(ours, ref, rtol=1e-12, atol=1e-14 * float(np.max(np.abs(ref))))


def test_gauss_nodes_symmetric_and_normalised():
    for n in (15, 94, 768):
        mu, w = gauss_nodes(n)
        assert np.all(np.diff(mu) > 0)
        np.testing.assert_array_equal(mu, -mu[::-1])
        assert abs(w.sum() - 2.0) < 1e-14


@pytest.mark.parametrize("case", ["vector_waist_t21.npz", "vector_waist_t62.npz"])
def test_oracle_vector_waist_halves_match_reference(case):
    """The two halves of the vector analysis (vector.py:75-166) on the
    reference's own waist of a stacked wind pair, and on the raw full-width
    zonal spectrum, against the reference's recorded outputs."""
    g = load_golden(case)
    o = _oracle_for(g)
    pair = np.stack([g["u"], g["v"]])
    _close(o.fourier(pair), g["waist"], 1e-15)
    z, d = o.vordiv_from_fourier(g["waist"])
    a = o.radius_m
    _close(z * a, g["zeta_waist"] * a, 1e-13)
    _close(d * a, g["div_waist"] * a, 1e-13)
    raw = np.fft.rfft(pair, axis=-1) / int(g["nlon"])
    z, d = o.vordiv_from_fourier(raw)
    _close(z * a, g["zeta_raw"] * a, 1e-13)
    _close(d * a, g["div_raw"] * a, 1e-13)
    _close(o.divergence_from_fourier(g["waist"]) * a, g["div_only"] * a, 1e-13)
    # the waist route and the whole-call route agree in the reference itself
    _close(g["zeta_waist"] * a, g["zeta"] * a, 1e-13)
