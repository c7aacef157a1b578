"""Seeded synthetic inputs for tests and benchmarks (host numpy).

Red-spectrum coefficients: ``c_nm = sigma_n (g1 + i g2)``, ``g ~ N(0, 1)``,
``sigma_n = (n (n + 1))^-1.5`` for ``n >= 1``, ``c_00 = 0``, ``Imag(c_n0) = 0``,
zero above the triangle.  Ensemble members add independent draws of the same
spectrum at a relative amplitude.  The Rossby-Haurwitz wave is the analytic
Williamson (1992) test-6 wind with wavenumber R.
"""
from __future__ import annotations

import math

import numpy as np

CONTROL_SEED = 20261203
EARTH_OMEGA = 7.292e-5


def red_spectrum(truncation: int, planes: int, seed: int = CONTROL_SEED) -> np.ndarray:
    t = int(truncation)
    rng = np.random.default_rng(seed)
    n = np.arange(t + 1, dtype=np.float64)
    sigma = np.zeros(t + 1)
    sigma[1:] = (n[1:] * (n[1:] + 1.0)) ** -1.5
    shape = (int(planes), t + 1, t + 1)
    c = sigma[:, None] * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    c *= np.tri(t + 1, dtype=bool)
    c[..., :, 0] = c[..., :, 0].real
    c[..., 0, 0] = 0.0
    return c


def ensemble_member(control: np.ndarray, member: int, amplitude: float = 0.1,
                    seed: int = CONTROL_SEED) -> np.ndarray:
    t = control.shape[-1] - 1
    pert = red_spectrum(t, control.shape[0], seed + 1000 + int(member))
    return control + amplitude * pert


def rossby_haurwitz_wind(mu: np.ndarray, nlon: int, *, omega=7.848e-6, k=7.848e-6, wavenumber=4,
                         radius_m=6_371_220.0):
    """Analytic (u, v) of the Rossby-Haurwitz wave on a Gaussian grid."""
    lat = np.arcsin(np.asarray(mu))[:, None]
    lon = (np.arange(nlon) * 2.0 * np.pi / nlon)[None, :]
    r = int(wavenumber)
    c, s = np.cos(lat), np.sin(lat)
    a = radius_m
    u = a * omega * c + a * k * c ** (r - 1) * (r * s * s - c * c) * np.cos(r * lon)
    v = -a * k * r * c ** (r - 1) * s * np.sin(r * lon)
    return u, v


def seeded_vertical_operator(nlev: int = 40, seed: int = CONTROL_SEED):
    """Seeded ``B`` (nlev x nlev+1) and ``C`` (nlev+1 x nlev) whose structure
    matrix ``M = -B C`` is symmetric and strictly diagonally dominant with a
    positive diagonal, so its modes are real and its eigenvalues positive.

    The diagonal holds gravity-wave speeds squared from 340 m/s (deepest
    mode) down to 8 m/s; each off-diagonal entry is a seeded fraction of the
    geometric mean of its two diagonal entries, scaled so every row's
    off-diagonal sum stays below half its diagonal.  ``C = [I; w^T]`` carries a
    seeded surface-pressure row ``w`` and ``B = [-M - b w^T | b]`` a seeded
    surface column ``b``, so ``-B C = M`` exactly.
    """
    rng = np.random.default_rng(seed + 40)
    speeds = np.geomspace(340.0, 8.0, int(nlev))
    diag = speeds ** 2
    off = rng.uniform(-1.0, 1.0, (nlev, nlev))
    off = 0.5 * (off + off.T)
    np.fill_diagonal(off, 0.0)
    off *= np.sqrt(np.outer(diag, diag))
    row = np.abs(off).sum(axis=1)
    scale = np.min(0.5 * diag / np.maximum(row, 1e-300))
    m = np.diag(diag) + off * min(1.0, scale)
    w = rng.uniform(0.5, 1.5, nlev) / nlev
    b = rng.uniform(-1.0, 1.0, nlev) * 1e-2
    b_matrix = np.concatenate([-m - np.outer(b, w), b[:, None]], axis=1)
    c_matrix = np.concatenate([np.eye(nlev), w[None, :]], axis=0)
    return b_matrix, c_matrix
