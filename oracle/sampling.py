"""CPU oracle of point sampling -- TEST INFRASTRUCTURE ONLY.

Imported by ``tests/`` as the checker; the product path
(``b200sht.sampling``) never imports it.  A numpy restatement of the
reference's host sampling path (spectral/sampling.py:382-515): the
orthonormal P_n^m(sin phi) and dP/dphi of ``oracle.dense_sht`` at the
points, per order the amplitudes sum_n c_nm P_nm, and
sum_m (m ? 2 : 1) Re(A_m e^{i m lambda}); the gradient's i m and dP/dphi
sums scaled by 1 / (a cos phi) and 1 / a.  Pinned against
``tests/golden/sampling_t21.npz`` (the reference's own sample_scalar /
sample_gradient / sample_wind, recorded by make_golden_sampling.py).
"""
from __future__ import annotations

import numpy as np

from oracle.dense_sht import legendre_derivative_table, legendre_table


def sample(coeff, lat_deg, lon_deg, *, gradient=False, radius=6371220.0):
    c = np.asarray(coeff, dtype=np.complex128)
    t = c.shape[-1] - 1
    lat = np.deg2rad(np.asarray(lat_deg, dtype=np.float64)).ravel()
    lon = np.deg2rad(np.asarray(lon_deg, dtype=np.float64)).ravel()
    p = legendre_table(t, np.sin(lat))
    d = legendre_derivative_table(t, np.sin(lat), p) if gradient else None
    lead = c.shape[:-2]
    out0 = np.zeros((*lead, lat.size))
    out1 = np.zeros_like(out0)
    for m in range(t + 1):
        phase = np.exp(1j * m * lon)
        mult = 1.0 if m == 0 else 2.0
        amp = np.einsum("...n,np->...p", c[..., m:, m], p[m:, m])
        if gradient:
            damp = np.einsum("...n,np->...p", c[..., m:, m], d[m:, m])
            out0 += mult * (1j * m * amp * phase).real
            out1 += mult * (damp * phase).real
        else:
            out0 += mult * (amp * phase).real
    if gradient:
        return out0 / (radius * np.cos(lat)), out1 / radius
    return out0


def inverse_laplacian(coeff, radius=6371220.0):
    c = np.asarray(coeff, dtype=np.complex128)
    n = np.arange(c.shape[-1])[:, None].astype(np.float64)
    eig = -n * (n + 1.0) / (radius * radius)
    out = np.where(n > 0, c / np.where(n > 0, eig, 1.0), 0.0)
    out[..., 0] = out[..., 0].real
    return out
