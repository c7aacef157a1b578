"""CPU oracle for the spherical-harmonic transform pair -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s ``cpu_baseline`` / ``--impl
reference`` leg may import it.  The CUDA library under ``gpuwm-global_b200/``
never calls into it and has no CPU fallback.

It is a float64 numpy restatement of the reference's dense transform
(FahrenheitResearch/gpuwm-global, ``tests/global_spectral_dense_reference.py``
and ``src/arwen_global/spectral/{grid,legendre,transform,vector}.py``), written
from the published algorithm:

* Gaussian grid: ``numpy.polynomial.legendre.leggauss`` nodes, ascending
  (row 0 southernmost), longitudes ``2*pi*i/nlon``
  (``src/arwen_global/spectral/grid.py:26-126``).
* Orthonormal associated Legendre values by the normalised three-term
  recurrence with the Condon-Shortley phase
  (``src/arwen_global/spectral/legendre.py:76-117``), and ``dP/dphi``
  (``legendre.py:120-146``).
* Analysis rows ``2*pi*w_j*P_nm(mu_j)`` Gram-solved per order
  (``src/arwen_global/spectral/transform.py:97-119``).
* forward = ``rfft/nlon`` cut to ``m <= T`` then the per-order contraction and
  ``Imag(c[:,0]) = 0`` (``transform.py:1294-1404``, ``1435-1490``);
  inverse = contraction then ``irfft(nlon * W)`` (``transform.py:1629-1746``).
* Gradient, zonal/meridional derivative, Laplacian, inverse Laplacian and
  projection (``transform.py:1124-1144``, ``1748-1811``).
* Vector operators by integration by parts (``src/arwen_global/spectral/vector.py:19-73``).

Parity pin: ``tests/golden/make_golden.py`` imports the reference itself (in
the build container, where its source tree is mounted) and records inputs
and outputs at small truncations in ``tests/golden/*.npz``;
``tests/test_oracle_golden.py`` holds this module to those fixtures.
"""
from __future__ import annotations

import math

import numpy as np

EARTH_RADIUS_M = 6_371_220.0  # src/arwen_global/spectral/constants.py:4


# --------------------------------------------------------------------- grid
def grid_shape(truncation, nlat=None, nlon=None, dealias_factor=1.5):
    """``(nlat, nlon)`` for a truncation (grid.py:26-94): the quadratic rule
    ``nlat >= ceil(f*(T+1))``, ``nlon >= ceil(2f*(T+1))`` rounded up to even;
    explicit sizes below the rule are refused."""
    t = int(truncation)
    if t < 1:
        raise ValueError(f"truncation must be >= 1, got {truncation}")
    req_lat = max(t + 1, int(math.ceil(dealias_factor * (t + 1))))
    req_lon = max(2 * t + 1, int(math.ceil(2.0 * dealias_factor * (t + 1))))
    if nlat is None:
        nl = req_lat
    else:
        nl = int(nlat)
        if nl < req_lat:
            raise ValueError(f"nlat={nl} is too small for T{t}; need at least {req_lat}")
    if nlon is None:
        no = req_lon + (req_lon % 2)
    else:
        no = int(nlon)
        if no % 2 or no < req_lon:
            raise ValueError(f"nlon={no} must be even and >= {req_lon}")
    return nl, no


def gauss_nodes(nlat):
    """Gauss-Legendre nodes ``mu`` (ascending) and weights (grid.py:112-125)."""
    mu, w = np.polynomial.legendre.leggauss(int(nlat))
    return mu.astype(np.float64), w.astype(np.float64)


# ------------------------------------------------------------------ legendre
def legendre_table(truncation, mu):
    """``P[n, m, j]``: orthonormal ``N_nm P_n^m(mu_j)``, zero where ``m > n``.

    Diagonal ``P_mm = -sqrt((2m+1)/(2m)) * sqrt(1-mu^2) * P_{m-1,m-1}`` from
    ``1/sqrt(4 pi)``; first off-diagonal ``P_{m+1,m} = sqrt(2m+3) mu P_mm``;
    then ``P_nm = a_nm (mu P_{n-1,m} - b_nm P_{n-2,m})`` with
    ``a = sqrt((4n^2-1)/(n^2-m^2))``, ``b = sqrt(((n-1)^2-m^2)/(4(n-1)^2-1))``
    (legendre.py:76-117).
    """
    t = int(truncation)
    x = np.asarray(mu, dtype=np.float64)
    p = np.zeros((t + 1, t + 1, x.size))
    root = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    p[0, 0] = 1.0 / math.sqrt(4.0 * math.pi)
    for m in range(1, t + 1):
        p[m, m] = -math.sqrt((2 * m + 1) / (2.0 * m)) * root * p[m - 1, m - 1]
    for m in range(t):
        p[m + 1, m] = math.sqrt(2 * m + 3) * x * p[m, m]
    for n in range(2, t + 1):
        ms = np.arange(0, n - 1)
        a = np.sqrt((4.0 * n * n - 1.0) / (n * n - ms * ms))
        b = np.sqrt(((n - 1.0) ** 2 - ms * ms) / (4.0 * (n - 1.0) ** 2 - 1.0))
        p[n, : n - 1] = a[:, None] * (x[None, :] * p[n - 1, : n - 1] - b[:, None] * p[n - 2, : n - 1])
    return p


def legendre_derivative_table(truncation, mu, p):
    """``dP/dphi[n, m, j] = cos(phi) (n mu P_nm - c_nm P_{n-1,m}) / (mu^2 - 1)``
    with ``c_nm = sqrt((n^2-m^2)(2n+1)/(2n-1))`` (legendre.py:120-146)."""
    t = int(truncation)
    x = np.asarray(mu, dtype=np.float64)
    denom = x * x - 1.0
    coslat = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    d = np.zeros_like(p)
    for n in range(1, t + 1):
        m = np.arange(0, n + 1)
        num = n * x[None, :] * p[n, : n + 1]
        c = np.sqrt((n * n - m[:n] ** 2) * (2.0 * n + 1.0) / (2.0 * n - 1.0))
        num[:n] -= c[:, None] * p[n - 1, :n]
        d[n, : n + 1] = coslat[None, :] * num / denom[None, :]
    return d


def gram_solved_analysis(p, w):
    """Analysis rows ``2 pi w P`` solved against the per-order Gram matrix
    (transform.py:97-119): ``A_m = solve(rows_m @ P_m^T, rows_m)``."""
    t1 = p.shape[0]
    rows_all = p * w[None, None, :] * (2.0 * math.pi)
    a = np.zeros_like(p)
    for m in range(t1):
        rows = rows_all[m:, m, :]
        gram = rows @ p[m:, m, :].T
        a[m:, m, :] = np.linalg.solve(gram, rows)
    return a


# ----------------------------------------------------------------- transform
class DenseSHT:
    """float64 dense transform on a Gaussian grid (the oracle).

    Spectral arrays are ``(*lead, T+1, T+1)`` complex indexed ``[n, m]``;
    grid arrays ``(*lead, nlat, nlon)`` real, row 0 southernmost.
    """

    def __init__(self, truncation, nlat=None, nlon=None, dealias_factor=1.5,
                 radius_m=EARTH_RADIUS_M, gram=True):
        self.truncation = int(truncation)
        self.nlat, self.nlon = grid_shape(truncation, nlat, nlon, dealias_factor)
        self.radius_m = float(radius_m)
        self.mu, self.w = gauss_nodes(self.nlat)
        self.coslat = np.sqrt(np.maximum(0.0, 1.0 - self.mu * self.mu))
        t1 = self.truncation + 1
        p = legendre_table(self.truncation, self.mu)
        d = legendre_derivative_table(self.truncation, self.mu, p)
        a = gram_solved_analysis(p, self.w) if gram else p * self.w * (2.0 * math.pi)
        # Order-leading layouts so each contraction is one batched matmul.
        self.basis_mnj = np.ascontiguousarray(p.transpose(1, 0, 2))
        self.dbasis_mnj = np.ascontiguousarray(d.transpose(1, 0, 2))
        self.analysis_mjn = np.ascontiguousarray(a.transpose(1, 2, 0))
        n = np.arange(t1, dtype=np.float64)
        self.lap_eigen = -(n * (n + 1.0)) / (self.radius_m ** 2)
        self.tri = np.tri(t1, dtype=bool)
        scale = 2.0 * math.pi / self.radius_m
        m = np.arange(t1, dtype=np.float64)
        self.rotation_weight = (1j * m)[None, :] * (self.w / self.coslat * scale)[:, None]
        self.shear_weight = (self.w * scale)[:, None]

    @property
    def spectral_shape(self):
        return (self.truncation + 1, self.truncation + 1)

    @property
    def grid_shape(self):
        return (self.nlat, self.nlon)

    # -- contraction: values[..., k, m] x table[m, k, n] -> out[..., n, m]
    @staticmethod
    def _contract(values, table):
        lead = values.shape[:-2]
        k, mcount = values.shape[-2:]
        stacked = np.moveaxis(values, -1, 0).reshape(mcount, -1, k)
        real = np.ascontiguousarray(stacked.real) @ table
        imag = np.ascontiguousarray(stacked.imag) @ table
        out = (real + 1j * imag).reshape(mcount, *lead, table.shape[-1])
        return np.moveaxis(out, 0, -1)

    def fourier(self, field):
        f = np.asarray(field, dtype=np.float64)
        return np.fft.rfft(f, axis=-1)[..., : self.truncation + 1] / self.nlon

    def forward(self, field):
        out = self._contract(self.fourier(field), self.analysis_mjn)
        out[..., :, 0] = out[..., :, 0].real
        return out

    def _synthesize(self, coeff, table_mnj):
        c = np.asarray(coeff, dtype=np.complex128)
        values = self._contract(c, table_mnj)
        spectrum = np.zeros((*c.shape[:-2], self.nlat, self.nlon // 2 + 1), np.complex128)
        spectrum[..., : self.truncation + 1] = self.nlon * values
        return np.fft.irfft(spectrum, n=self.nlon, axis=-1)

    def inverse(self, coeff):
        return self._synthesize(coeff, self.basis_mnj)

    def inverse_meridional_derivative(self, coeff):
        return self._synthesize(coeff, self.dbasis_mnj)

    def inverse_zonal_derivative(self, coeff):
        m = 1j * np.arange(self.truncation + 1)
        return self.inverse(np.asarray(coeff) * m)

    def gradient(self, coeff):
        east = self.inverse_zonal_derivative(coeff) / (self.radius_m * self.coslat[:, None])
        north = self.inverse_meridional_derivative(coeff) / self.radius_m
        return east, north

    def project(self, coeff):
        c = np.array(coeff, dtype=np.complex128, copy=True)
        c *= self.tri
        c[..., :, 0] = c[..., :, 0].real
        return c

    def laplacian(self, coeff):
        return np.asarray(coeff, dtype=np.complex128) * self.lap_eigen[:, None]

    def inverse_laplacian(self, coeff):
        c = np.asarray(coeff, dtype=np.complex128)
        out = np.zeros_like(c)
        out[..., 1:, :] = c[..., 1:, :] / self.lap_eigen[1:, None]
        return self.project(out)

    # -- vector (vector.py:36-73)
    def wind_from_vordiv(self, vorticity, divergence):
        psi = self.inverse_laplacian(vorticity)
        chi = self.inverse_laplacian(divergence)
        east, north = self.gradient(np.stack([psi, chi]))
        return -north[0] + east[1], east[0] + north[1]

    def vordiv_from_wind(self, u, v):
        return self.vordiv_from_fourier(
            self.fourier(np.stack([np.asarray(u, np.float64), np.asarray(v, np.float64)])))

    def vordiv_from_fourier(self, fourier):
        """The contraction half of the vector analysis on a stacked (u, v)
        waist, or on a wider zonal spectrum cut here (vector.py:113-134)."""
        fm = np.asarray(fourier, dtype=np.complex128)[..., : self.truncation + 1]
        basis_mjn = self.basis_mnj.transpose(0, 2, 1)
        dbasis_mjn = self.dbasis_mnj.transpose(0, 2, 1)
        rot = self._contract(fm * self.rotation_weight, basis_mjn)
        shear = self._contract(fm * self.shear_weight, dbasis_mjn)
        return self.project(rot[1] + shear[0]), self.project(rot[0] - shear[1])

    def divergence_from_fourier(self, fourier):
        """D = i m rot[u] - shear[v] alone (vector.py:136-166)."""
        fm = np.asarray(fourier, dtype=np.complex128)[..., : self.truncation + 1]
        rot = self._contract(fm[0] * self.rotation_weight, self.basis_mnj.transpose(0, 2, 1))
        shear = self._contract(fm[1] * self.shear_weight, self.dbasis_mnj.transpose(0, 2, 1))
        return self.project(rot - shear)

    # -- diagnostics (transform.py:1813-1863)
    def spectral_weights(self):
        wt = np.ones(self.truncation + 1)
        wt[1:] = 2.0
        return wt

    def global_mean(self, field):
        return 0.5 * np.sum(np.asarray(field, np.float64).mean(axis=-1) * self.w, axis=-1)

    def transform_check(self, seed=0, max_degree=None):
        rng = np.random.default_rng(seed)
        t = self.truncation if max_degree is None else min(self.truncation, int(max_degree))
        coeff = np.zeros(self.spectral_shape, np.complex128)
        for n in range(t + 1):
            for m in range(n + 1):
                coeff[n, m] = rng.normal() + (0.0j if m == 0 else 1j * rng.normal())
        grid = self.inverse(coeff)
        back = self.forward(grid)
        scale = max(1.0, float(np.max(np.abs(coeff))))
        spatial = self.global_mean(grid ** 2)
        spectral = float(np.sum(np.abs(coeff) ** 2 * self.spectral_weights()[None, :]) / (4 * np.pi))
        return {
            "roundtrip_relative_linf": float(np.max(np.abs(back - coeff)) / scale),
            "parseval_relative_error": abs(spatial - spectral) / max(1.0, abs(spectral)),
        }


# ----------------------------------------------------------------- Helmholtz
def helmholtz_inverse(eigenvalues, eigenvectors, k2, dt_s, alpha=1.0):
    """``(I + (alpha dt)^2 k_n^2 M)^-1`` per degree through the modal
    decomposition ``V diag(1/(1 + s lambda_j)) V^-1``; identity at ``k = 0``
    (src/arwen_global/semi_implicit.py:585-609)."""
    scale = (float(alpha) * float(dt_s)) ** 2 * np.asarray(k2, np.float64)
    modal = 1.0 / (1.0 + scale[:, None] * np.asarray(eigenvalues)[None, :])
    vinv = np.linalg.inv(eigenvectors)
    inv = np.einsum("ij,nj,jk->nik", eigenvectors, modal, vinv)
    inv[np.asarray(k2) == 0.0] = np.eye(len(eigenvalues))
    return inv


def solve_shifted(divergence, theta, lnps, b_matrix, c_matrix, eigenvalues,
                  eigenvectors, tau_w, radius_m=EARTH_RADIUS_M):
    """``(I - tau w L) y = r`` per total degree (semi_implicit.py:921-953 and
    the ``_finish`` pin/project of 815-843).

    ``divergence``/``theta``: ``(nlev, T+1, T+1)`` complex; ``lnps``:
    ``(T+1, T+1)``.  Returns ``(divergence, theta, lnps)`` projected, with
    degree zero passed through."""
    t1 = divergence.shape[-1]
    n = np.arange(t1, dtype=np.float64)
    k2 = n * (n + 1.0) / radius_m ** 2
    inv = helmholtz_inverse(eigenvalues, eigenvectors, k2, tau_w, 1.0)
    x = np.concatenate([theta, lnps[None]], axis=0)
    forcing = divergence + tau_w * k2[None, :, None] * np.einsum("ij,jnm->inm", b_matrix, x)
    d_new = np.einsum("nij,jnm->inm", inv, forcing)
    x_new = x + tau_w * np.einsum("ij,jnm->inm", c_matrix, d_new)
    d_new[:, 0, 0] = divergence[:, 0, 0]
    x_new[:, 0, 0] = x[:, 0, 0]
    tri = np.tri(t1, dtype=bool)

    def proj(c):
        c = c * tri
        c[..., :, 0] = c[..., :, 0].real
        return c

    return proj(d_new), proj(x_new[:-1]), proj(x_new[-1])


def _finish(divergence, x, d_new, x_new):
    """Degree zero passes through, the max divergence increment, projection
    (semi_implicit.py:815-843)."""
    t1 = divergence.shape[-1]
    d_new = np.array(d_new)
    x_new = np.array(x_new)
    d_new[:, 0, 0] = divergence[:, 0, 0]
    x_new[:, 0, 0] = x[:, 0, 0]
    metric = float(np.max(np.abs(d_new - divergence)))
    tri = np.tri(t1, dtype=bool)

    def proj(c):
        c = c * tri
        c[..., :, 0] = c[..., :, 0].real
        return c

    return proj(d_new), proj(x_new[:-1]), proj(x_new[-1]), metric


def _wave_k2(t1, radius_m):
    n = np.arange(t1, dtype=np.float64)
    return n * (n + 1.0) / radius_m ** 2


def apply_crank_nicolson(divergence, theta, lnps, b_matrix, c_matrix, eigenvalues, eigenvectors,
                         dt_w, alpha, radius_m=EARTH_RADIUS_M):
    """The off-centred Crank-Nicolson step of the subtracted operator
    (semi_implicit.py:887-919): ``forcing = D + dt k^2 B x - a(1-a) dt^2 k^2 M D``,
    ``D' = (I + (a dt)^2 k^2 M)^-1 forcing``, ``x' = x + dt C((1-a) D + a D')``.
    Returns ``(divergence, theta, lnps, max |D' - D|)``."""
    k2 = _wave_k2(divergence.shape[-1], radius_m)
    structure = -b_matrix @ c_matrix
    inv = helmholtz_inverse(eigenvalues, eigenvectors, k2, dt_w, alpha)
    x = np.concatenate([theta, lnps[None]], axis=0)
    kc = k2[None, :, None]
    forcing = (divergence + dt_w * kc * np.einsum("ij,jnm->inm", b_matrix, x)
               - (alpha * (1.0 - alpha) * dt_w * dt_w) * kc
               * np.einsum("ij,jnm->inm", structure, divergence))
    d_new = np.einsum("nij,jnm->inm", inv, forcing)
    x_new = x + dt_w * np.einsum("ij,jnm->inm", c_matrix,
                                 (1.0 - alpha) * divergence + alpha * d_new)
    return _finish(divergence, x, d_new, x_new)


def half_map_scalars(frequencies, dt_s, alpha):
    """``(p, q)`` with ``sqrt(g) = p + i q omega`` for the off-centred
    Crank-Nicolson factor ``g = (1 + i(1-a) omega dt) / (1 - i a omega dt)``
    (principal root); ``omega = 0`` gives ``p = 1, q = dt/2``
    (semi_implicit.py:611-627)."""
    y = frequencies * float(dt_s)
    root = np.sqrt((1.0 + 1j * (1.0 - alpha) * y) / (1.0 - 1j * alpha * y))
    safe = np.where(frequencies > 0.0, frequencies, 1.0)
    return root.real, np.where(frequencies > 0.0, root.imag / safe, 0.5 * float(dt_s))


def linear_tendencies(divergence, theta, lnps, b_matrix, c_matrix, weight,
                      radius_m=EARTH_RADIUS_M):
    """``w L y`` (semi_implicit.py:796-813): ``D_t = w k^2 (B x)`` and
    ``x_t = w (C D)`` with ``x = (theta, ln ps)``, each projected.  Returns
    ``(divergence_t, theta_t, lnps_t)``."""
    t1 = divergence.shape[-1]
    k2 = _wave_k2(t1, radius_m)
    x = np.concatenate([theta, lnps[None]], axis=0)
    d_t = weight * k2[None, :, None] * np.einsum("ij,jnm->inm", b_matrix, x)
    x_t = weight * np.einsum("ij,jnm->inm", c_matrix, divergence)
    tri = np.tri(t1, dtype=bool)

    def proj(c):
        c = c * tri
        c[..., :, 0] = c[..., :, 0].real
        return c

    return proj(d_t), proj(x_t[:-1]), proj(x_t[-1])


def half_apply(divergence, theta, lnps, b_matrix, c_matrix, eigenvalues, eigenvectors,
               x_eigenvalues, x_eigenvectors, dt_w, alpha, radius_m=EARTH_RADIUS_M):
    """The square root ``H = P + Q L`` of the Crank-Nicolson map, per block
    and degree (semi_implicit.py:629-663, 845-877):
    ``D' = P_D D + Q_D k^2 B x``, ``x' = P_x x + Q_x C D``, with
    ``P_D = V diag(p) V^-1`` at frequencies ``k sqrt(lambda)`` and ``P_x``,
    ``Q_x`` in the modes of ``C B`` at ``k sqrt(-mu)``."""
    k2 = _wave_k2(divergence.shape[-1], radius_m)
    k = np.sqrt(k2)
    p_d, q_d = half_map_scalars(k[:, None] * np.sqrt(eigenvalues)[None, :], dt_w, alpha)
    p_x, q_x = half_map_scalars(k[:, None] * np.sqrt(-np.asarray(x_eigenvalues))[None, :],
                                dt_w, alpha)
    v, vi = eigenvectors, np.linalg.inv(eigenvectors)
    w, wi = x_eigenvectors, np.linalg.inv(x_eigenvectors)
    maps = [np.einsum("ij,nj,jk->nik", a, s, b) for a, s, b in
            ((v, p_d, vi), (v, q_d, vi), (w, p_x, wi), (w, q_x, wi))]
    x = np.concatenate([theta, lnps[None]], axis=0)
    l_div = k2[None, :, None] * np.einsum("ij,jnm->inm", b_matrix, x)
    l_x = np.einsum("ij,jnm->inm", c_matrix, divergence)
    d_new = (np.einsum("nij,jnm->inm", maps[0], divergence)
             + np.einsum("nij,jnm->inm", maps[1], l_div))
    x_new = np.einsum("nij,jnm->inm", maps[2], x) + np.einsum("nij,jnm->inm", maps[3], l_x)
    return _finish(divergence, x, d_new, x_new)
