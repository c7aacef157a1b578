"""Record golden vectors of point sampling from the reference.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden_sampling.py <reference checkout>

It builds the reference's numpy T21 transform and runs its own
``sample_scalar``, ``sample_gradient`` and ``sample_wind``
(``arwen_global.spectral.sampling``, the host path) on seeded coefficients
(two fields) at seeded points (the exact poles included for the scalar),
and writes ``tests/golden/sampling_t21.npz``.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path.insert(0, str(Path(ref_root) / "src"))
    from arwen_global.spectral.sampling import sample_gradient, sample_scalar, sample_wind
    from arwen_global.spectral.transform import SphericalHarmonicTransform

    T = 21
    t = SphericalHarmonicTransform.create(T)
    rng = np.random.default_rng(20261203)
    n = np.arange(T + 1)[:, None]
    m = np.arange(T + 1)[None, :]
    sigma = np.where(n >= 1, (np.maximum(n, 1) * (n + 1.0)) ** -0.5, 0.0)
    c = (rng.standard_normal((2, T + 1, T + 1)) + 1j * rng.standard_normal((2, T + 1, T + 1)))
    c = np.where(m <= n, c * sigma, 0.0)
    c[..., 0] = c[..., 0].real
    lat = np.concatenate([[-90.0, 90.0], rng.uniform(-89.0, 89.0, 40)])
    lon = rng.uniform(-180.0, 540.0, lat.size)
    scalar = sample_scalar(t, c, lat, lon)
    east, north = sample_gradient(t, c, lat[2:], lon[2:])
    u, v = sample_wind(t, c[0], c[1], lat[2:], lon[2:])
    np.savez_compressed(HERE / "sampling_t21.npz", coeff=c, lat=lat, lon=lon, scalar=scalar,
                        east=east, north=north, u=u, v=v, radius=np.float64(t.grid.radius_m))
    print("wrote", HERE / "sampling_t21.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])
