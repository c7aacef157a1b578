"""Point sampling on the GPU (sht_sample) against the reference's recorded
host path and the oracle.  FP64: 1e-12 of the field's magnitude."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - b)) / np.max(np.abs(b)))


def test_sampling_matches_reference(golden):
    from b200sht import SphericalHarmonicTransform
    from b200sht.sampling import sample_gradient, sample_scalar, sample_wind

    g = golden("sampling_t21.npz")
    t = SphericalHarmonicTransform.create(21, precision="float64")
    c = torch.as_tensor(g["coeff"], device="cuda")
    assert _rel(sample_scalar(t, c, g["lat"], g["lon"]), g["scalar"]) < 1e-12
    e, n = sample_gradient(t, c, g["lat"][2:], g["lon"][2:])
    assert _rel(e, g["east"]) < 1e-12 and _rel(n, g["north"]) < 1e-12
    u, v = sample_wind(t, c[0], c[1], g["lat"][2:], g["lon"][2:])
    assert _rel(u, g["u"]) < 1e-12 and _rel(v, g["v"]) < 1e-12


@pytest.mark.parametrize("T", [62, 255])
def test_sampling_against_oracle_and_grid(T):
    """Random points at T62 and T255 (fields > 4: more than one pass), and
    at the transform's own grid points the synthesis's values."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.sampling import sample_scalar
    from b200sht.synthetic import red_spectrum
    from oracle import sampling as O

    t = SphericalHarmonicTransform.create(T, precision="float64")
    c = red_spectrum(T, 5, 11)
    rng = np.random.default_rng(T)
    lat = rng.uniform(-90, 90, 64)
    lon = rng.uniform(0, 360, 64)
    got = sample_scalar(t, torch.as_tensor(c, device="cuda"), lat, lon)
    assert got.shape == (5, 64)
    assert _rel(got, O.sample(c, lat, lon)) < 1e-12
    grid = t.backend.to_numpy(t.inverse(torch.as_tensor(c, device="cuda")))
    la = np.rad2deg(t.grid.lat_rad)[:: max(1, t.grid.nlat // 8)]
    lo = np.rad2deg(t.grid.lon_rad)[:: max(1, t.grid.nlon // 8)]
    lo2, la2 = np.meshgrid(lo, la)
    pts = sample_scalar(t, torch.as_tensor(c, device="cuda"), la2, lo2)
    ref = grid[:, :: max(1, t.grid.nlat // 8), :: max(1, t.grid.nlon // 8)]
    assert _rel(pts, ref) < 1e-11


def test_sampling_errors_and_device_output(golden):
    from b200sht import SphericalHarmonicTransform
    from b200sht.sampling import regular_latlon_scalar, sample_gradient, sample_scalar

    g = golden("sampling_t21.npz")
    t = SphericalHarmonicTransform.create(21, precision="float64")
    c = torch.as_tensor(g["coeff"], device="cuda")
    with pytest.raises(ValueError, match="exact poles"):
        sample_gradient(t, c, [90.0], [0.0])
    with pytest.raises(ValueError, match="latitude must lie"):
        sample_scalar(t, c, [91.0], [0.0])
    with pytest.raises(ValueError, match="finite"):
        sample_scalar(t, c, [np.nan], [0.0])
    with pytest.raises(ValueError, match="chunk_points"):
        sample_scalar(t, c, [0.0], [0.0], chunk_points=0)
    out = sample_scalar(t, c, g["lat"], g["lon"], as_device=True)
    assert isinstance(out, torch.Tensor) and out.is_cuda
    lat, lon, f = regular_latlon_scalar(t, c[0], nlat=8, nlon=16)
    assert f.shape == (8, 16) and lat.shape == (8,) and lon.shape == (16,)


@pytest.mark.parametrize("T", [1, 3, 7])
def test_sampling_small_truncations(T):
    """Truncations with fewer orders than the kernel has order bands (some
    bands empty) and point counts that are not a multiple of 32: scalar and
    gradient against the oracle."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.sampling import sample_gradient, sample_scalar
    from b200sht.synthetic import red_spectrum
    from oracle import sampling as O

    t = SphericalHarmonicTransform.create(T, precision="float64")
    c = red_spectrum(T, 3, 5 + T)
    rng = np.random.default_rng(T)
    lat = rng.uniform(-85, 85, 37)
    lon = rng.uniform(0, 360, 37)
    dc = torch.as_tensor(c, device="cuda")
    assert _rel(sample_scalar(t, dc, lat, lon), O.sample(c, lat, lon)) < 1e-12
    e, n = sample_gradient(t, dc, lat, lon)
    we, wn = O.sample(c, lat, lon, gradient=True)
    assert _rel(e, we) < 1e-12 and _rel(n, wn) < 1e-12


@pytest.mark.parametrize("T", [7, 21])
def test_packed_basis_blocks(T):
    """The reference's packed-basis form (sampling.py:198-254): the blocks
    against the oracle's recurrence entry by entry, [Re c | Im c] @ B against
    the sampled field and gradient, and the FP32 blocks as the FP64 ones
    rounded once."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.sampling import (packed_basis, packed_coefficients, sample_gradient,
                                  sample_scalar, triangle_index)
    from b200sht.synthetic import red_spectrum
    from oracle import sampling as O
    from oracle.dense_sht import legendre_derivative_table, legendre_table

    t = SphericalHarmonicTransform.create(T, precision="float64")
    rng = np.random.default_rng(100 + T)
    lat_d = rng.uniform(-85, 85, 45)
    lon_d = rng.uniform(0, 360, 45)
    lat, lon = np.deg2rad(lat_d), np.deg2rad(lon_d)
    b = packed_basis(torch, T, lat, lon, gradient=False).cpu().numpy()
    bz, bm = (x.cpu().numpy() for x in packed_basis(torch, T, lat, lon, gradient=True))
    k = (T + 1) * (T + 2) // 2
    assert b.shape == bz.shape == bm.shape == (2 * k, lat.size)
    n_idx, m_idx = triangle_index(T)
    mu = np.sin(lat)
    p = legendre_table(T, mu)[n_idx, m_idx]            # (K, points)
    dp = legendre_derivative_table(T, mu, legendre_table(T, mu))[n_idx, m_idx]
    mult = np.where(m_idx == 0, 1.0, 2.0)[:, None]
    ang = m_idx[:, None] * lon[None, :]
    want = np.concatenate([mult * p * np.cos(ang), -(mult * p * np.sin(ang))])
    assert np.max(np.abs(b - want)) <= 1e-13 * np.max(np.abs(want))
    mm = mult * m_idx[:, None]
    want_z = np.concatenate([-(mm * p * np.sin(ang)), -(mm * p * np.cos(ang))])
    want_m = np.concatenate([mult * dp * np.cos(ang), -(mult * dp * np.sin(ang))])
    assert np.max(np.abs(bz - want_z)) <= 1e-13 * np.max(np.abs(want_z))
    assert np.max(np.abs(bm - want_m)) <= 1e-13 * np.max(np.abs(want_m))
    # the contraction of the packed spectrum with the blocks is the sample
    c = red_spectrum(T, 3, 7 + T)
    pc, lead = packed_coefficients(torch, c, T)
    assert lead == (3,) and tuple(pc.shape) == (3, 2 * k)
    pc = pc.cpu().numpy()
    dc = torch.as_tensor(c, device="cuda")
    assert _rel(pc @ b, sample_scalar(t, dc, lat_d, lon_d)) < 1e-12
    assert _rel(pc @ b, O.sample(c, lat_d, lon_d)) < 1e-12
    a = t.grid.radius_m
    e, nrt = sample_gradient(t, dc, lat_d, lon_d)
    assert _rel(pc @ bz / (a * np.cos(lat)), e) < 1e-12 and _rel(pc @ bm / a, nrt) < 1e-12
    # FP32 blocks: the FP64 values rounded once
    b32 = packed_basis(torch, T, lat, lon, gradient=False, dtype=np.float32).cpu().numpy()
    assert b32.dtype == np.float32 and np.array_equal(b32, b.astype(np.float32))
