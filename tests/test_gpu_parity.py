"""Parity of the CUDA path against the reference's recorded outputs and the
CPU oracle.

Bars: FP64 path within 1e-12 (relative to the largest output value) of the
reference; FP32 and split-FP16 paths within 2e-6 relative spectral L2 (the
reference's Parseval weights, transform.py:1813-1825) and 2e-6 relative max
grid error.  Every call goes through the C ABI (``libb200sht.so``).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["sht_t9.npz", "sht_t21.npz", "sht_t31_wide.npz", "sht_t62.npz"]
PRECISIONS = ["float64", "float32", "split16"]


def _tol(precision):
    return 1e-12 if precision == "float64" else 2e-6


def _make(g, precision):
    from b200sht import SphericalHarmonicTransform

    return SphericalHarmonicTransform.create(
        int(g["truncation"]), nlat=int(g["nlat"]), nlon=int(g["nlon"]),
        dealias_factor=float(g["dealias_factor"]), precision=precision)


def rel_l2(a, b):
    t1 = a.shape[-1]
    w = np.where(np.arange(t1) == 0, 1.0, 2.0)[None, :]
    return float(np.sqrt(np.sum(w * np.abs(a - b) ** 2) / np.sum(w * np.abs(b) ** 2)))


def rel_max(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", autouse=True)
def _built():
    from b200sht import build

    build.build()


@pytest.mark.parametrize("case", CASES)
def test_geometry_matches_leggauss(case):
    """Nodes within 2 ulp of the reference's leggauss nodes; weights within
    leggauss's own error (its polar weights are off by up to 1.3e-12 at 94
    latitudes against 40-digit values); both checked tightly against the
    40-digit fixture."""
    g = load_golden(case)
    sht = _make(g, "float64")
    n = int(g["nlat"])
    exact = load_golden("gauss_exact.npz")
    np.testing.assert_allclose(sht.grid.sin_lat, g["mu"], rtol=0, atol=2.3e-16)
    np.testing.assert_allclose(sht.grid.quadrature_weights, g["weights"], rtol=3e-12, atol=0)
    np.testing.assert_allclose(sht.grid.sin_lat, exact[f"mu_{n}"], rtol=0, atol=2.3e-16)
    np.testing.assert_allclose(sht.grid.quadrature_weights, exact[f"w_{n}"], rtol=2e-13, atol=0)
    assert np.all(np.diff(sht.grid.sin_lat) > 0)


def test_geometry_t511_against_exact():
    from b200sht import GaussianGrid

    grid = GaussianGrid.create(511)
    exact = load_golden("gauss_exact.npz")
    assert grid.shape == (768, 1536)
    np.testing.assert_allclose(grid.sin_lat, exact["mu_768"], rtol=0, atol=2.3e-16)
    np.testing.assert_allclose(grid.quadrature_weights, exact["w_768"], rtol=2e-11, atol=0)
    assert abs(grid.quadrature_weights.sum() - 2.0) < 1e-14


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("case", CASES)
def test_scalar_transforms_match_reference(case, precision):
    g = load_golden(case)
    sht = _make(g, precision)
    tol = _tol(precision)
    np_ = sht.backend.to_numpy
    fwd = np_(sht.forward(g["grid"]))
    if precision == "float64":
        assert rel_max(fwd, g["forward"]) < tol
    else:
        assert rel_l2(fwd, g["forward"]) < tol
    assert np.all(fwd[..., 0].imag == 0)
    assert np.all(np.triu(np.ones(fwd.shape[-2:]), 1)[None] * fwd == 0)
    assert rel_max(np_(sht.inverse(g["coeff"])), g["inverse"]) < tol
    assert rel_max(np_(sht.inverse_zonal_derivative(g["coeff"])), g["zonal"]) < tol
    assert rel_max(np_(sht.inverse_meridional_derivative(g["coeff"])), g["meridional"]) < tol
    east, north = sht.gradient(g["coeff"])
    assert rel_max(np_(east), g["east"]) < tol
    assert rel_max(np_(north), g["north"]) < tol
    assert rel_max(np_(sht.laplacian(g["coeff"])), g["laplacian"]) < tol
    assert rel_max(np_(sht.inverse_laplacian(g["coeff"])), g["inverse_laplacian"]) < tol
    proj = np_(sht.project(g["project_in"]))
    if precision == "float64":
        np.testing.assert_array_equal(proj, g["project_out"])
    else:
        assert rel_max(proj, g["project_out"]) < 1e-7
    sht.check_device()


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("case", CASES)
def test_vector_transforms_match_reference(case, precision):
    from b200sht import VorticityDivergenceOperator

    g = load_golden(case)
    sht = _make(g, precision)
    vec = VorticityDivergenceOperator(sht)
    tol = _tol(precision)
    np_ = sht.backend.to_numpy
    u, v = vec.wind_from_vordiv(g["coeff"], g["coeff2"])
    assert rel_max(np_(u), g["wind_u"]) < tol
    assert rel_max(np_(v), g["wind_v"]) < tol
    z, d = vec.vordiv_from_wind(g["u"], g["v"])
    z, d = np_(z), np_(d)
    if precision == "float64":
        assert rel_max(z, g["vort"]) < tol
        assert rel_max(d, g["div"]) < tol
    else:
        assert rel_l2(z, g["vort"]) < tol
        assert rel_l2(d, g["div"]) < tol
    assert np.all(z[..., 0, 0] == 0) and np.all(d[..., 0, 0] == 0)
    sht.check_device()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_transform_check_roundtrip_and_parseval(precision):
    from b200sht import SphericalHarmonicTransform

    for t in (15, 170):
        sht = SphericalHarmonicTransform.create(t, precision=precision)
        r = sht.transform_check(seed=7)
        if precision == "float64":
            assert r["roundtrip_relative_linf"] < 5e-13
            assert r["parseval_relative_error"] < 5e-14
        else:
            assert r["roundtrip_relative_linf"] < 5e-5
            assert r["parseval_relative_error"] < 1e-5


def test_closed_form_harmonics_fp64():
    """Analysis of fields built from closed forms, with no inverse() in the
    path (the reference's known-answer test)."""
    from b200sht import SphericalHarmonicTransform

    sht = SphericalHarmonicTransform.create(15, precision="float64")
    lat, lon = sht.grid.mesh()
    s, c = np.sin(lat), np.cos(lat)
    harmonics = {
        (0, 0): np.full(lat.shape, 1 / math.sqrt(4 * math.pi)),
        (1, 0): math.sqrt(3 / (4 * math.pi)) * s,
        (2, 0): math.sqrt(5 / (16 * math.pi)) * (3 * s ** 2 - 1),
        (2, 2): 2 * np.real(math.sqrt(15 / (32 * math.pi)) * c ** 2 * np.exp(2j * lon)),
        (3, 2): 2 * np.real(math.sqrt(105 / (32 * math.pi)) * s * c ** 2 * np.exp(2j * lon)),
    }
    for (n, m), f in harmonics.items():
        coeff = sht.backend.to_numpy(sht.forward(f))
        assert abs(coeff[n, m] - 1.0) < 1e-14
        coeff[n, m] = 0
        assert np.max(np.abs(coeff)) < 1e-14


def test_vector_known_answers_fp64():
    from b200sht import SphericalHarmonicTransform, VorticityDivergenceOperator
    from b200sht.synthetic import red_spectrum

    sht = SphericalHarmonicTransform.create(15, precision="float64")
    vec = VorticityDivergenceOperator(sht)
    np_ = sht.backend.to_numpy
    # Solid-body rotation: zeta = 2 u0 sin(phi) / a, no divergence.
    u0 = 40.0
    u = u0 * sht.grid.cos_lat[:, None] * np.ones((1, sht.grid.nlon))
    z, d = vec.vordiv_from_wind(u, np.zeros_like(u))
    zg = np_(sht.inverse(z))
    expected = 2 * u0 * sht.grid.sin_lat[:, None] / sht.grid.radius_m
    assert np.max(np.abs(zg - expected)) < 2e-18
    assert np.max(np.abs(np_(sht.inverse(d)))) < 2e-18
    # Round trip of a low-degree (vorticity, divergence) pair.
    c = red_spectrum(15, 2, seed=3)
    c[..., 10:, :] = 0
    uu, vv = vec.wind_from_vordiv(c[0], c[1])
    z2, d2 = vec.vordiv_from_wind(uu, vv)
    assert np.max(np.abs(np_(z2) - c[0])) < 2e-12 * max(1.0, np.max(np.abs(c)))
    assert np.max(np.abs(np_(d2) - c[1])) < 2e-12 * max(1.0, np.max(np.abs(c)))


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("case", ["helmholtz_t7_l6.npz", "helmholtz_t21_l40.npz"])
def test_helmholtz_matches_reference(case, precision):
    from b200sht import SphericalHarmonicTransform, VerticalModeOperator, VerticalModeSemiImplicit

    g = load_golden(case)
    sht = SphericalHarmonicTransform.create(int(g["truncation"]), precision=precision)
    op = VerticalModeOperator(g["b_matrix"], g["c_matrix"], g["eigenvalues"], g["eigenvectors"])
    semi = VerticalModeSemiImplicit(divergence_weight=float(g["weight"]))
    d, th, lp = semi.solve_arrays(sht, op, float(g["tau_s"]), g["divergence"], g["theta"], g["lnps"])
    tol = 1e-11 if precision == "float64" else 2e-5
    np_ = sht.backend.to_numpy
    assert rel_max(np_(d), g["out_divergence"]) < tol
    assert rel_max(np_(th), g["out_theta"]) < tol
    assert rel_max(np_(lp), g["out_lnps"]) < tol


def test_shape_errors_use_reference_wording():
    from b200sht import SphericalHarmonicTransform

    sht = SphericalHarmonicTransform.create(9, precision="float64")
    with pytest.raises(ValueError, match="grid field has trailing shape"):
        sht.forward(np.zeros((3, 4)))
    with pytest.raises(ValueError, match="spectral field has trailing shape"):
        sht.inverse(np.zeros((3, 4), complex))


def test_leading_shapes_and_empty_batches():
    from b200sht import SphericalHarmonicTransform
    from oracle.dense_sht import DenseSHT

    sht = SphericalHarmonicTransform.create(21, precision="float64")
    ora = DenseSHT(21)
    rng = np.random.default_rng(0)
    for lead in [(), (3,), (2, 5)]:
        f = rng.standard_normal((*lead, sht.grid.nlat, sht.grid.nlon))
        c = sht.backend.to_numpy(sht.forward(f))
        assert c.shape == (*lead, 22, 22)
        assert rel_max(c, ora.forward(f)) < 1e-12
    empty = sht.forward(np.zeros((0, sht.grid.nlat, sht.grid.nlon)))
    assert tuple(empty.shape) == (0, 22, 22)


CONFIG_GRIDS = [(62, 94, 192, 1.49), (126, 192, 384, 1.5), (255, 384, 768, 1.5),
                (511, 768, 1536, 1.5)]


@pytest.mark.parametrize("t,nlat,nlon,df", CONFIG_GRIDS)
def test_fp32_and_split_against_fp64_at_config_grids(t, nlat, nlon, df):
    """Every transform of the FP32 and split paths, with the register-resident
    FFT and with the generic FFT, against the GPU FP64 path (itself pinned to
    the reference above and to the oracle below)."""
    import torch

    from b200sht import SphericalHarmonicTransform, VorticityDivergenceOperator
    from b200sht._lib import SHT_FLAG_GENERIC_FFT
    from b200sht.synthetic import red_spectrum

    import json

    from conftest import GOLDEN

    kw = dict(nlat=nlat, nlon=nlon, dealias_factor=df)
    # The reference's own float32 vector analysis loses digits to the
    # i m rot + shear cancellation (1.9e-6 at T62 to 1.2e-5 at T511): the
    # vorticity/divergence bar is 1.5x the reference float32 error for the
    # FP32 path and 2x for the split path (whose two FP16 terms per operand
    # carry 22 bits, one fewer than FP32).
    ref_err = json.loads((GOLDEN / "reference_fp32_errors.json").read_text())[str(t)]
    vordiv_tol = {"float32": max(2e-6, 1.5 * ref_err["vordiv"]),
                  "split16": max(2e-6, 2.0 * ref_err["vordiv"])}
    coeff = red_spectrum(t, 3)
    f64 = SphericalHarmonicTransform.create(t, precision="float64", **kw)
    vec64 = VorticityDivergenceOperator(f64)
    np_ = f64.backend.to_numpy
    g64 = f64.inverse(coeff)
    c64 = np_(f64.forward(g64))
    e64, n64 = (np_(x) for x in f64.gradient(coeff))
    u64, v64 = (np_(x) for x in vec64.wind_from_vordiv(coeff, coeff[::-1].copy()))
    z64, d64 = (np_(x) for x in vec64.vordiv_from_wind(u64, v64))
    for precision in ("float32", "split16"):
        for flags in (0, SHT_FLAG_GENERIC_FFT):
            sht = SphericalHarmonicTransform.create(t, precision=precision, plan_flags=flags, **kw)
            vec = VorticityDivergenceOperator(sht)
            tag = (precision, flags)
            g32 = g64.to(torch.float32)
            err = rel_l2(np_(sht.forward(g32)), c64)
            assert err < 2e-6, (tag, "forward", err)
            err = rel_max(np_(sht.inverse(coeff)), np_(g64))
            assert err < 2e-6, (tag, "inverse", err)
            e, n = sht.gradient(coeff)
            err = max(rel_max(np_(e), e64), rel_max(np_(n), n64))
            assert err < 2e-6, (tag, "gradient", err)
            u, v = vec.wind_from_vordiv(coeff, coeff[::-1].copy())
            err = max(rel_max(np_(u), u64), rel_max(np_(v), v64))
            assert err < 2e-6, (tag, "wind", err)
            z, d = vec.vordiv_from_wind(u64, v64)
            err = max(rel_l2(np_(z), z64), rel_l2(np_(d), d64))
            assert err < vordiv_tol[precision], (tag, "vordiv", err)
            sht.check_device()


def test_fp64_against_oracle_t255():
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    ora = DenseSHT(255)
    sht = SphericalHarmonicTransform.create(255, precision="float64")
    coeff = red_spectrum(255, 2, seed=5)
    g = sht.backend.to_numpy(sht.inverse(coeff))
    assert rel_max(g, ora.inverse(coeff)) < 1e-12
    rng = np.random.default_rng(1)
    f = g + 0.01 * rng.standard_normal(g.shape)
    assert rel_max(sht.backend.to_numpy(sht.forward(f)), ora.forward(f)) < 1e-12


def test_fp64_roundtrip_t511():
    """forward(inverse(c)) = c at full size (the Gram-corrected analysis)."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    sht = SphericalHarmonicTransform.create(511, precision="float64")
    coeff = red_spectrum(511, 2, seed=9)
    back = sht.backend.to_numpy(sht.forward(sht.inverse(coeff)))
    assert rel_l2(back, coeff) < 1e-12
    assert rel_max(back, coeff) < 1e-11


def test_t511_against_oracle_two_planes():
    """The benchmark's grid (T511, 768 x 1536) against the CPU oracle itself
    on two planes: FP64 within 1e-12, FP32 and split16 within 2e-6
    (forward: relative spectral L2; inverse: max grid error)."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    ora = DenseSHT(511)
    coeff = red_spectrum(511, 2, seed=11)
    want_g = ora.inverse(coeff)
    want_c = ora.forward(want_g)
    for precision, tol in (("float64", 1e-12), ("float32", 2e-6), ("split16", 2e-6)):
        sht = SphericalHarmonicTransform.create(511, precision=precision)
        np_ = sht.backend.to_numpy
        g = want_g if precision == "float64" else want_g.astype(np.float32)
        assert rel_l2(np_(sht.forward(g)), want_c) < tol, precision
        assert rel_max(np_(sht.inverse(coeff)), want_g) < tol, precision
        sht.check_device()


def test_baseline_configs_at_full_plane_counts():
    """The first two benchmark configurations at their full plane counts
    (40 levels x 4 fields + ln ps = 161 planes): T62 on the 94 x 192 grid in
    FP64 against the oracle on every plane (forward, inverse, and u, v from
    vorticity/divergence on the 40 levels), and T255 on 384 x 768 in FP32
    against the FP64 plan on every plane."""
    from b200sht import SphericalHarmonicTransform, VorticityDivergenceOperator
    from b200sht.synthetic import red_spectrum
    from oracle.dense_sht import DenseSHT

    planes = 40 * 4 + 1
    sht = SphericalHarmonicTransform.create(62, nlat=94, nlon=192, dealias_factor=1.49,
                                            precision="float64")
    ora = DenseSHT(62, 94, 192, dealias_factor=1.49)
    np_ = sht.backend.to_numpy
    coeff = red_spectrum(62, planes, seed=11)
    grid = ora.inverse(coeff)
    assert rel_max(np_(sht.inverse(coeff)), grid) < 1e-12
    assert rel_l2(np_(sht.forward(grid)), ora.forward(grid)) < 1e-12
    vec = VorticityDivergenceOperator(sht)
    u, v = (np_(x) for x in vec.wind_from_vordiv(coeff[:40], coeff[40:80]))
    uo, vo = ora.wind_from_vordiv(coeff[:40], coeff[40:80])
    assert rel_max(u, uo) < 1e-12 and rel_max(v, vo) < 1e-12

    t64 = SphericalHarmonicTransform.create(255, precision="float64")
    t32 = SphericalHarmonicTransform.create(255, precision="float32")
    c = red_spectrum(255, planes, seed=12)
    g64 = t64.inverse(c)
    assert rel_max(np_(t32.inverse(c)), np_(g64)) < 2e-6
    assert rel_l2(t32.backend.to_numpy(t32.forward(g64.float())),
                  np_(t64.forward(g64))) < 2e-6
    t32.check_device()
