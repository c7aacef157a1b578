"""Spectral scalars, gradients and winds at arbitrary latitude/longitude
points, on the GPU.

Mirrors the reference's ``arwen_global.spectral.sampling`` public functions
(``sample_scalar``, ``sample_gradient``, ``sample_wind``,
``regular_latlon_coordinates``, ``regular_latlon_scalar``;
sampling.py:346-571) with the same arguments, shapes and error texts; the
evaluation runs in ``libb200sht.so`` (``sht_sample``: one CTA per point,
the orthonormal recurrence in FP64 with the reference's operand order).
Results come back as numpy arrays, or as CUDA tensors with
``as_device=True``.  ``precision`` accepts the reference's two names; the
evaluation is FP64 for both (its float32 mode rounds the basis to float32
to save GEMM time, which this direct evaluator has no use for).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

SAMPLE_PRECISIONS = ("float64", "float32")
_SAMPLERS: dict = {}


def _sampler(truncation: int, device: torch.device):
    key = (int(truncation), device.index)
    h = _SAMPLERS.get(key)
    if h is None:
        h = ctypes.c_void_p()
        with torch.cuda.device(device):
            _lib.call("sht_sampler_create", int(truncation), ctypes.byref(h))
        _SAMPLERS[key] = h
    return h


def _resolve_precision(precision) -> str:
    p = "float64" if precision is None else precision
    if p not in SAMPLE_PRECISIONS:
        raise ValueError(f"precision must be one of {SAMPLE_PRECISIONS}, got {precision!r}")
    return p


def _points(latitude_deg, longitude_deg):
    lat, lon = np.broadcast_arrays(np.asarray(latitude_deg, dtype=np.float64),
                                   np.asarray(longitude_deg, dtype=np.float64))
    if not np.isfinite(lat).all() or not np.isfinite(lon).all():
        raise ValueError("sample coordinates must be finite")
    if np.any((lat < -90.0) | (lat > 90.0)):
        raise ValueError("latitude must lie in [-90, 90] degrees")
    return np.deg2rad(lat.ravel()), np.deg2rad(lon.ravel()), lat.shape


def _coefficients(transform, coeff):
    dev = transform.backend.device
    c = torch.as_tensor(coeff, device=dev) if not isinstance(coeff, torch.Tensor) else coeff.to(dev)
    if not torch.is_complex(c):
        c = c.to(torch.complex128)
    transform._validate_spectral(c)
    lead = tuple(c.shape[:-2])
    t1 = transform.truncation + 1
    cmn = c.to(torch.complex128).reshape(-1, t1, t1).transpose(-1, -2).contiguous()
    return cmn, lead


def _run(transform, coeff, latitude_deg, longitude_deg, gradient, precision, as_device):
    _resolve_precision(precision)
    cmn, lead = _coefficients(transform, coeff)
    lat, lon, point_shape = _points(latitude_deg, longitude_deg)
    if gradient and np.any(np.abs(np.cos(lat)) < 1.0e-12):
        raise ValueError("vector/gradient sampling is undefined at the exact poles")
    dev = cmn.device
    fields, npts = cmn.shape[0], lat.size
    lat_t = torch.as_tensor(lat, device=dev)
    lon_t = torch.as_tensor(lon, device=dev)
    out0 = torch.empty((fields, npts), dtype=torch.float64, device=dev)
    out1 = torch.empty_like(out0) if gradient else None
    sample_into(transform.truncation, cmn, lat_t, lon_t, float(transform.grid.radius_m), out0,
                out1)
    shape = (*lead, *point_shape)
    res = [o.reshape(shape) for o in ((out0, out1) if gradient else (out0,))]
    if not as_device:
        res = [o.cpu().numpy() for o in res]
    return tuple(res) if gradient else res[0]


def sample_into(truncation: int, coeff_mn: torch.Tensor, lat_rad: torch.Tensor,
                lon_rad: torch.Tensor, radius: float, out0: torch.Tensor, out1=None) -> None:
    """The kernel alone: coeff_mn complex128 (fields, m, n) contiguous,
    lat/lon float64 radians, out0 (and out1 for the gradient) float64
    (fields, npoints)."""
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    _lib.call("sht_sample", _sampler(truncation, coeff_mn.device), ptr(coeff_mn),
              coeff_mn.shape[0], lat_rad.numel(), ptr(lat_rad), ptr(lon_rad),
              0 if out1 is None else 1, float(radius), ptr(out0), ptr(out1),
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def sample_scalar(transform, coeff, latitude_deg, longitude_deg, *, chunk_points=None,
                  precision=None, as_device=False):
    """Synthesize one or more real scalar fields at arbitrary points (leading
    coefficient dimensions retained; exact poles admitted)."""
    _chunk(chunk_points)
    return _run(transform, coeff, latitude_deg, longitude_deg, False, precision, as_device)


def sample_gradient(transform, coeff, latitude_deg, longitude_deg, *, chunk_points=None,
                    precision=None, as_device=False):
    """Physical eastward/northward gradient at non-polar points."""
    _chunk(chunk_points)
    return _run(transform, coeff, latitude_deg, longitude_deg, True, precision, as_device)


def sample_wind(transform, vorticity, divergence, latitude_deg, longitude_deg, *,
                chunk_points=None, precision=None, as_device=False):
    """Invert vorticity/divergence and sample the eastward/northward wind."""
    psi = transform.inverse_laplacian(vorticity)
    chi = transform.inverse_laplacian(divergence)
    pe, pn = sample_gradient(transform, psi, latitude_deg, longitude_deg,
                             chunk_points=chunk_points, precision=precision, as_device=as_device)
    ce, cn = sample_gradient(transform, chi, latitude_deg, longitude_deg,
                             chunk_points=chunk_points, precision=precision, as_device=as_device)
    return -pn + ce, pe + cn


def _chunk(requested):
    """The reference's host path chunks points to bound its workspace; the
    device evaluator needs no chunks, but the argument is validated alike."""
    if requested is not None:
        if isinstance(requested, bool) or not isinstance(requested, (int, np.integer)) \
                or int(requested) < 1:
            raise ValueError("chunk_points must be a positive integer")


def regular_latlon_coordinates(nlat: int, nlon: int, *, include_poles: bool = False):
    """Cell-centre regular global coordinates, or pole-inclusive latitudes."""
    if isinstance(nlat, bool) or isinstance(nlon, bool):
        raise ValueError("regular-grid dimensions must be integers")
    ny, nx = int(nlat), int(nlon)
    if ny != nlat or nx != nlon:
        raise ValueError("regular-grid dimensions must be integers")
    if ny < 2 or nx < 4:
        raise ValueError("regular grid needs nlat>=2 and nlon>=4")
    if include_poles:
        lat = np.linspace(-90.0, 90.0, ny, dtype=np.float64)
    else:
        lat = -90.0 + (np.arange(ny, dtype=np.float64) + 0.5) * 180.0 / ny
    lon = np.arange(nx, dtype=np.float64) * 360.0 / nx
    return lat, lon


def regular_latlon_scalar(transform, coeff, *, nlat: int, nlon: int, include_poles: bool = False,
                          chunk_points=None):
    lat, lon = regular_latlon_coordinates(nlat, nlon, include_poles=include_poles)
    lon2, lat2 = np.meshgrid(lon, lat)
    return lat, lon, sample_scalar(transform, coeff, lat2, lon2, chunk_points=chunk_points)


# ------------------------------------------------- the packed basis form
def triangle_index(truncation: int) -> tuple[np.ndarray, np.ndarray]:
    """``(n, m)`` of every coefficient inside the triangle, order-major
    (``m = 0..T``, ``n = m..T`` inside each order): the packed order of
    ``packed_basis`` and ``packed_coefficients`` (sampling.py:72-80)."""
    t = int(truncation)
    ms = np.concatenate([np.full(t + 1 - m, m, dtype=np.int64) for m in range(t + 1)])
    ns = np.concatenate([np.arange(m, t + 1, dtype=np.int64) for m in range(t + 1)])
    return ns, ms


def _torch_dtype(dtype) -> torch.dtype:
    if dtype in (torch.float64, torch.float32):
        return dtype
    d = np.dtype(dtype)
    if d == np.float64:
        return torch.float64
    if d == np.float32:
        return torch.float32
    raise ValueError(f"dtype must be float64 or float32, got {dtype!r}")


def packed_basis(xp, truncation: int, lat_rad, lon_rad, *, gradient: bool, dtype=np.float64,
                 device=None):
    """The packed real basis blocks of a point chunk on the device
    (sampling.py:198-237): scalar, one ``(2K, p)`` block ``B`` with
    ``[Re c | Im c] @ B`` the field (``B[k] = mult P cos(m lam)``,
    ``B[K + k] = -mult P sin(m lam)``); gradient, the zonal and meridional
    blocks, whose products over ``a cos(phi)`` and ``a`` are the eastward
    and northward derivatives.  ``K = (T+1)(T+2)/2`` in the order of
    ``triangle_index``; one kernel (``sht_sample_packed_basis``).  ``xp`` is
    accepted for the reference's signature; the blocks are CUDA tensors."""
    t = int(truncation)
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    lat = torch.as_tensor(np.asarray(lat_rad, dtype=np.float64).ravel(), device=dev)
    lon = torch.as_tensor(np.asarray(lon_rad, dtype=np.float64).ravel(), device=dev)
    if lat.numel() != lon.numel():
        raise ValueError("lat_rad and lon_rad must hold the same number of points")
    npts = int(lat.numel())
    ktri = (t + 1) * (t + 2) // 2
    tdt = _torch_dtype(dtype)
    code = _lib.SHT_PREC_F64 if tdt == torch.float64 else _lib.SHT_PREC_F32
    b0 = torch.empty((2 * ktri, npts), dtype=tdt, device=dev)
    b1 = torch.empty_like(b0) if gradient else None
    ptr = lambda x: ctypes.c_void_p(x.data_ptr()) if x is not None else None
    with torch.cuda.device(dev):
        _lib.call("sht_sample_packed_basis", _sampler(t, dev), npts, ptr(lat), ptr(lon),
                  1 if gradient else 0, code, ptr(b0), ptr(b1),
                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return (b0, b1) if gradient else b0


def packed_coefficients(xp, coeff, truncation: int, dtype=np.float64):
    """``[Re c | Im c]`` of ``coeff (..., T+1, T+1)`` over the packed
    triangle, ``(fields, 2K)`` in ``dtype`` with the leading dimensions
    flattened, and the leading shape (sampling.py:240-254).  A CUDA tensor
    stays on its device; anything else is read as host data."""
    t = int(truncation)
    c = coeff if isinstance(coeff, torch.Tensor) else torch.as_tensor(np.asarray(coeff))
    lead = tuple(c.shape[:-2])
    fields = int(np.prod(lead)) if lead else 1
    n_idx, m_idx = triangle_index(t)
    tri = torch.as_tensor(n_idx * (t + 1) + m_idx, device=c.device)
    flat = c.reshape(fields, (t + 1) * (t + 1))[:, tri]
    tdt = _torch_dtype(dtype)
    packed = torch.empty((fields, 2 * int(tri.numel())), dtype=tdt, device=c.device)
    if torch.is_complex(flat):
        packed[:, :tri.numel()] = flat.real
        packed[:, tri.numel():] = flat.imag
    else:
        packed[:, :tri.numel()] = flat
        packed[:, tri.numel():] = 0
    return packed, lead
