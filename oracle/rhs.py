"""CPU oracle of the fused RHS kernels -- TEST INFRASTRUCTURE ONLY.

Imported by ``tests/`` and ``bench.py``'s CPU legs as the checker; the
product path (``b200sht.rhs``) never imports it.  numpy restatements of the
specifications the reference's CuPy kernels (spectral/fused.py:233-386)
replace, in their association:

* momentum/Bernoulli and the tracer-flux pair and scalar tendency
  (dynamics.py:1436-1489 and 1592-1610, restated from the numpy branches);
* the van Leer limited vertical flux divergence (dynamics.py:1355-1434).

The vertical flux divergence is pinned to the reference's own numpy method
run on seeded columns (``tests/golden/rhs_vertical_flux.npz``); the three
elementwise chains are pinned, bit for bit, to the reference's numpy
specifications of its fused kernels (``tools/gpu_selftest_rhs.py``:
``momentum_bernoulli_reference``, ``tracer_flux_reference``,
``scalar_tendency_reference``) run on seeded fields
(``tests/golden/rhs_elementwise.npz``).  Both fixtures are recorded by
``tests/golden/make_golden_rhs.py``.
"""
from __future__ import annotations

import numpy as np


def momentum_bernoulli(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, rgas):
    av = zeta + cor
    pf = rgas * tv * pg
    mu = av * v - wu - pf * ge
    mv = -av * u - wv - pf * gn
    bern = 0.5 * (u ** 2 + v ** 2) + phi
    return mu, mv, bern


def tracer_flux(dp, s, u, v):
    m = dp * s
    return m * u, m * v


def scalar_tendency(h, vert, s, dpt, dp):
    return (-h - vert - s * dpt) / dp


def vertical_flux_divergence(s, w, pf, ph):
    """Upstream van Leer face values at the interfaces, bounded by the two
    adjacent layers; out = flux[k+1] - flux[k] with zero boundary fluxes."""
    nlev = pf.shape[0]
    grad = np.zeros_like(s)
    ga = (s[..., 1:-1, :, :] - s[..., :-2, :, :]) / (pf[1:-1] - pf[:-2])
    gb = (s[..., 2:, :, :] - s[..., 1:-1, :, :]) / (pf[2:] - pf[1:-1])
    prod = ga * gb
    mono = prod > 0.0
    grad[..., 1:-1, :, :] = np.where(mono, 2.0 * prod / np.where(mono, ga + gb, 1.0), 0.0)
    if nlev >= 2:
        grad[..., 0, :, :] = (s[..., 1, :, :] - s[..., 0, :, :]) / (pf[1] - pf[0])
        grad[..., -1, :, :] = (s[..., -1, :, :] - s[..., -2, :, :]) / (pf[-1] - pf[-2])
    wi = w[1:nlev]
    above, below = s[..., :-1, :, :], s[..., 1:, :, :]
    from_above = above + grad[..., :-1, :, :] * (ph[1:nlev] - pf[:-1])
    from_below = below + grad[..., 1:, :, :] * (ph[1:nlev] - pf[1:])
    face = np.where(wi >= 0.0, from_above, from_below)
    face = np.minimum(np.maximum(face, np.minimum(above, below)), np.maximum(above, below))
    flux = np.zeros((*s.shape[:-3], nlev + 1, *s.shape[-2:]), dtype=s.dtype)
    flux[..., 1:nlev, :, :] = wi * face
    return flux[..., 1:, :, :] - flux[..., :-1, :, :]


def column_state(nlev, nlat, nlon, ntr, seed, dtype=np.float64):
    """Seeded hybrid-like columns: increasing full and half pressures,
    an interface pressure velocity of both signs (zero at the boundaries),
    and `ntr` tracers with smooth profiles, noise and sharp features."""
    rng = np.random.default_rng(seed)
    eta = (np.arange(nlev + 1) / nlev) ** 1.5
    ps = 1.0e5 + 2.0e3 * rng.standard_normal((nlat, nlon))
    ph = 1.0e3 + eta[:, None, None] * (ps[None] - 1.0e3)
    pf = np.sqrt(ph[:-1] * ph[1:])
    w = 0.5 * rng.standard_normal((nlev + 1, nlat, nlon))
    w[0] = 0.0
    w[-1] = 0.0
    k = np.arange(nlev)[:, None, None]
    s = np.stack([np.cos(0.3 * (t + 1) * k) + 0.2 * rng.standard_normal((nlev, nlat, nlon))
                  + (rng.random((nlev, nlat, nlon)) < 0.05) * 3.0 for t in range(ntr)])
    return (s.astype(dtype), w.astype(dtype), pf.astype(dtype), ph.astype(dtype))
