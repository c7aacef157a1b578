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
