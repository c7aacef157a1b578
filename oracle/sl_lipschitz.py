"""Oracle: the trajectory deformation diagnostics of the semi-Lagrangian step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports this module; the
tests use it as the checker of the CUDA kernel (``sht_sl_lipschitz``).

A numpy restatement of the reference's ``semilag.trajectory.lipschitz``
on its numpy path (src/arwen_global/semilag/trajectory.py:1174-1420): the
derivatives of the Cartesian wind components and of the level rate
(zonal centred differences, the non-uniform three-point latitude formula
with the pole reflection, vertical centred differences with one-sided ends;
trajectory.py:672-752), the closed-form norms of the flow Jacobian projected
on the local tangent basis (``_norms_reference``, trajectory.py:1038-1097,
with the symmetric 2x2 and 3x3 top eigenvalues of 621-669), the fold
determinants ``det(I + c J)`` (``_fold_reference``, 1140-1171) and the
reductions (maxima of the norms, minima of the two determinants and where
they sit).  Every array is in the caller's dtype and every scalar enters
as the reference's numpy expressions have it, so float32 inputs give the
reference's float32 numbers.  Pinned to the reference's own outputs by
``tests/golden/make_golden_lipschitz.py``.
"""
from __future__ import annotations

import math

import numpy as np


def _d_dlam(f, dlam):
    return (np.roll(f, -1, axis=2) - np.roll(f, 1, axis=2)) / (2.0 * dlam)


def _d_dk(f):
    out = np.empty_like(f)
    out[1:-1] = 0.5 * (f[2:] - f[:-2])
    out[0] = f[1] - f[0]
    out[-1] = f[-1] - f[-2]
    return out


def _rows_with_neighbours(field, nlat, nlon, held0, a0, a1):
    """Rows ``[a0, a1)`` of ``field`` (which holds rows ``[held0, held0 +
    field.shape[1])``) with one neighbour row each side: the held row next
    to them, or at a pole the pole row itself read half a turn round.
    Raises LookupError when a needed neighbour is not held."""
    lo, hi = a0 - held0, a1 - held0
    if a0 == 0:
        top = np.roll(field[:, lo:lo + 1, :], nlon // 2, axis=2)
    else:
        if lo < 1:
            raise LookupError("the row above the band is not held")
        top = field[:, lo - 1:lo, :]
    if a1 == nlat:
        bot = np.roll(field[:, hi - 1:hi, :], nlon // 2, axis=2)
    else:
        if hi + 1 > field.shape[1]:
            raise LookupError("the row below the band is not held")
        bot = field[:, hi:hi + 1, :]
    return np.concatenate([top, field[:, lo:hi, :], bot], axis=1)


def _d_dphi(field, lat_ext, nlat, nlon, held0, a0, a1):
    ext = _rows_with_neighbours(field, nlat, nlon, held0, a0, a1)
    n = a1 - a0
    x0 = lat_ext[a0 + 1:a0 + n + 1][None, :, None]
    x1 = lat_ext[a0 + 2:a0 + n + 2][None, :, None]
    x2 = lat_ext[a0 + 3:a0 + n + 3][None, :, None]
    f0, f1, f2 = ext[:, :-2, :], ext[:, 1:-1, :], ext[:, 2:, :]
    return (f0 * (x1 - x2) / ((x0 - x1) * (x0 - x2))
            + f1 * (2.0 * x1 - x0 - x2) / ((x1 - x0) * (x1 - x2))
            + f2 * (x1 - x0) / ((x2 - x0) * (x2 - x1)))


def _sym2_top(a00, a01, a11):
    half = 0.5 * (a00 + a11)
    rad = np.sqrt(np.maximum(0.25 * (a00 - a11) ** 2 + a01 * a01, 0.0))
    return half + rad


def _sym3_top(a00, a01, a02, a11, a12, a22):
    """Largest eigenvalue of a symmetric 3x3 by the trigonometric solution of
    its characteristic cubic, scaled to unit trace first (trajectory.py:621-663)."""
    trace = a00 + a11 + a22
    tiny = np.asarray(float(np.finfo(trace.dtype).eps), dtype=trace.dtype)
    scale = np.maximum(trace, tiny)
    inv = 1.0 / scale
    a00, a01, a02 = a00 * inv, a01 * inv, a02 * inv
    a11, a12, a22 = a11 * inv, a12 * inv, a22 * inv
    q = (a00 + a11 + a22) / 3.0
    b00, b11, b22 = a00 - q, a11 - q, a22 - q
    p2 = (b00 * b00 + b11 * b11 + b22 * b22
          + 2.0 * (a01 * a01 + a02 * a02 + a12 * a12)) / 6.0
    p = np.sqrt(np.maximum(p2, 0.0))
    safe = np.maximum(p, tiny)
    det = (b00 * (b11 * b22 - a12 * a12)
           - a01 * (a01 * b22 - a12 * a02)
           + a02 * (a01 * a12 - b11 * a02))
    r = np.clip(det / (2.0 * safe * safe * safe), -1.0, 1.0)
    return scale * (q + 2.0 * p * np.cos(np.arccos(r) / 3.0))


def _project(basis, vec):
    return basis[0] * vec[0] + basis[1] * vec[1] + basis[2] * vec[2]


def norms(dv, ds, sph, cph, sla, cla, lref):
    """(spectral, frobenius, horizontal, balanced) per point."""
    ex = (-sla, cla, np.zeros_like(sla))
    ey = (-sph * cla, -sph * sla, cph)
    dvdx, dvdy, dvdk = dv
    dsdx, dsdy, dsdk = ds
    j00, j01 = _project(ex, dvdx), _project(ex, dvdy)
    j02 = _project(ex, dvdk) / lref
    j10, j11 = _project(ey, dvdx), _project(ey, dvdy)
    j12 = _project(ey, dvdk) / lref
    j20, j21, j22 = lref * dsdx, lref * dsdy, dsdk
    frob = np.sqrt(j00 * j00 + j01 * j01 + j02 * j02 + j10 * j10 + j11 * j11 + j12 * j12
                   + j20 * j20 + j21 * j21 + j22 * j22)
    h00 = j00 * j00 + j10 * j10
    h11 = j01 * j01 + j11 * j11
    h01 = j00 * j01 + j10 * j11
    horizontal = np.sqrt(np.maximum(_sym2_top(h00, h01, h11), 0.0))
    spectral = np.sqrt(np.maximum(_sym3_top(
        h00 + j20 * j20, j00 * j01 + j10 * j11 + j20 * j21, j00 * j02 + j10 * j12 + j20 * j22,
        h11 + j21 * j21, j01 * j02 + j11 * j12 + j21 * j22, j02 * j02 + j12 * j12 + j22 * j22),
        0.0))
    # the coupling blocks rescaled to the geometric mean of their magnitudes
    e0, e1 = j02 * lref, j12 * lref
    d0, d1 = dsdx, dsdy
    emag = np.sqrt(e0 * e0 + e1 * e1)
    dmag = np.sqrt(d0 * d0 + d1 * d1)
    gmean = np.sqrt(emag * dmag)
    se = np.where(emag > 0.0, gmean / np.where(emag > 0.0, emag, 1.0), 0.0)
    sd = np.where(dmag > 0.0, gmean / np.where(dmag > 0.0, dmag, 1.0), 0.0)
    c02, c12, c20, c21 = e0 * se, e1 * se, d0 * sd, d1 * sd
    balanced = np.sqrt(np.maximum(_sym3_top(
        h00 + c20 * c20, j00 * j01 + j10 * j11 + c20 * c21, j00 * c02 + j10 * c12 + c20 * j22,
        h11 + c21 * c21, j01 * c02 + j11 * c12 + c21 * j22, c02 * c02 + c12 * c12 + j22 * j22),
        0.0))
    return spectral, frob, horizontal, balanced


def fold(dv, ds, sph, cph, sla, cla, c):
    """det(I + c J) per point."""
    ex = (-sla, cla, np.zeros_like(sla))
    ey = (-sph * cla, -sph * sla, cph)
    dvdx, dvdy, dvdk = dv
    dsdx, dsdy, dsdk = ds
    m00 = 1.0 + c * _project(ex, dvdx)
    m01 = c * _project(ex, dvdy)
    m02 = c * _project(ex, dvdk)
    m10 = c * _project(ey, dvdx)
    m11 = 1.0 + c * _project(ey, dvdy)
    m12 = c * _project(ey, dvdk)
    m20, m21, m22 = c * dsdx, c * dsdy, 1.0 + c * dsdk
    return (m00 * (m11 * m22 - m12 * m21) - m01 * (m10 * m22 - m12 * m20)
            + m02 * (m10 * m21 - m11 * m20))


def lipschitz(wind, lat_ext_host, nlon, radius_m, dt_s, *, extrapolated=None,
              reference_length_m=None, held=None, arrival=None, extrapolated_held=None):
    """The diagnostics of ``wind`` = (vx, vy, vz, level_rate), each
    ``(nlev, rows held, nlon)``.  ``held``/``arrival`` are row ranges
    ``(start, stop)`` of a band (default the whole grid); an
    ``extrapolated`` wind holds ``extrapolated_held`` rows.  Returns a dict:
    the five maxima, the two minimum determinants and the flat
    (level, arrival row, lon) index of each minimum."""
    wind = [np.asarray(f) for f in wind]
    dtype = wind[0].dtype
    nlev = wind[0].shape[0]
    nlat = len(lat_ext_host) - 4
    held = (0, nlat) if held is None else tuple(held)
    arrival = (0, nlat) if arrival is None else tuple(arrival)
    a0, a1 = arrival
    dlam = 2.0 * math.pi / nlon
    lref = radius_m * dlam if reference_length_m is None else float(reference_length_m)
    lat = np.asarray(lat_ext_host[2:nlat + 2], dtype=dtype)[None, :, None]
    lon = np.asarray(np.arange(nlon) * dlam, dtype=dtype)[None, None, :]
    lat_ext = np.asarray(lat_ext_host, dtype=dtype)
    sph, cph = np.sin(lat)[:, a0:a1], np.cos(lat)[:, a0:a1]
    sla, cla = np.sin(lon), np.cos(lon)
    inv_x = 1.0 / (radius_m * np.maximum(cph, dtype.type(1e-12)))
    inv_y = dtype.type(1.0 / radius_m)
    half = 0.5 * float(dt_s)

    def derivatives(flow, rows_held):
        own = slice(a0 - rows_held[0], a1 - rows_held[0])
        comps, rate = flow[:3], flow[3]
        dvdx = [inv_x * _d_dlam(c[:, own], dlam) for c in comps]
        dvdy = [inv_y * _d_dphi(c, lat_ext, nlat, nlon, rows_held[0], a0, a1) for c in comps]
        dvdk = [_d_dk(c[:, own]) for c in comps]
        ds = (inv_x * _d_dlam(rate[:, own], dlam),
              inv_y * _d_dphi(rate, lat_ext, nlat, nlon, rows_held[0], a0, a1),
              _d_dk(rate[:, own]))
        return (dvdx, dvdy, dvdk), ds

    dv, ds = derivatives(wind, held)
    spectral, frob, horizontal, balanced = norms(dv, ds, sph, cph, sla, cla, lref)
    dep = fold(dv, ds, sph, cph, sla, cla, dtype.type(+half))
    if extrapolated is None:
        arr = fold(dv, ds, sph, cph, sla, cla, dtype.type(-half))
    else:
        ex = [np.asarray(f) for f in extrapolated]
        ex_held = held if extrapolated_held is None else tuple(extrapolated_held)
        dve, dse = derivatives(ex, ex_held)
        arr = fold(dve, dse, sph, cph, sla, cla, dtype.type(-half))
    return {
        "spectral": float(np.max(spectral)), "frobenius": float(np.max(frob)),
        "horizontal": float(np.max(horizontal)), "vertical": float(np.max(np.abs(ds[2]))),
        "balanced": float(np.max(balanced)),
        "fold_departure": float(np.min(dep)), "fold_arrival": float(np.min(arr)),
        "where_departure": int(np.argmin(dep)), "where_arrival": int(np.argmin(arr)),
        "reference_length_m": lref, "shape": (nlev, a1 - a0, nlon),
    }


def level_rate_from_mass_flux(omega_half, p_full):
    """The vertical rate in level indices per second at full levels from the
    interface mass flux (trajectory.py:121-155)."""
    nlev = int(p_full.shape[0])
    s_half = np.zeros_like(omega_half)
    s_half[1:nlev] = omega_half[1:nlev] / (p_full[1:] - p_full[:-1])
    return 0.5 * (s_half[:nlev] + s_half[1:nlev + 1])


def deforming_wind(lat, nlon, nlev, *, speed=40.0, noise=120.0, seed=0, dtype=np.float64):
    """A seeded smooth wind with strain strong enough to fold at long steps:
    (vx, vy, vz, level_rate), each (nlev, nlat, nlon)."""
    rng = np.random.default_rng(seed)
    lat = np.asarray(lat, dtype=np.float64)[None, :, None]
    lon = (np.arange(nlon) * (2.0 * np.pi / nlon))[None, None, :]
    lev = np.arange(nlev, dtype=np.float64)[:, None, None]
    a, b = rng.uniform(0.5, 1.5, 2)
    u = speed * np.cos(lat) + noise * np.cos(lat) ** 2 * np.sin(2 * lon + a) * np.cos(lev / 3.0)
    v = noise * np.cos(lat) * np.sin(lat) * np.cos(3 * lon + b) * (1 + 0.1 * lev)
    w = 1e-4 * np.sin(lon + lat) * np.sin(np.pi * (lev + 0.5) / nlev)
    sph, cph = np.sin(lat), np.cos(lat)
    sla, cla = np.sin(lon), np.cos(lon)
    vx = -u * sla - v * sph * cla
    vy = u * cla - v * sph * sla
    vz = v * cph + 0.0 * u
    shape = (nlev, lat.shape[1], nlon)
    return tuple(np.array(np.broadcast_to(f, shape), dtype=dtype) for f in (vx, vy, vz, w))


def where_text(flat, shape, lat_ext_host, nlon, a0=0):
    """The reference's location text of a flat (level, row, lon) index
    (trajectory.py:1381-1390)."""
    _, nr, nl = shape
    kk, jj, ii = flat // (nr * nl), (flat // nl) % nr, flat % nl
    lat_d = float(np.degrees(lat_ext_host[jj + a0 + 2]))
    lon_d = float(np.degrees(ii * (2.0 * math.pi / nlon)))
    return f"level {kk}, lat {lat_d:.2f}, lon {lon_d:.2f}"
