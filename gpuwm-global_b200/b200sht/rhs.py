"""Fused right-hand-side kernels of the dycore step, on the GPU.

The reference keeps four CuPy elementwise kernels for the chains that
consume the synthesis output (spectral/fused.py:233-386:
``momentum_bernoulli_kernel``, ``tracer_flux_kernel``,
``scalar_tendency_kernel``, ``vertical_flux_divergence_kernel``), each the
replacement of a numpy expression in ``MoistHybridModel``
(dynamics.py:1355-1490, 1575-1610).  These functions take CUDA tensors
(float32 or float64, C-order ``(..., nlev, nlat, nlon)``) and run the
library's fused kernels (``sht_rhs_*``): the elementwise three as 16-byte
vector streams, the vertical flux divergence as one thread per column
marching down the levels.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

_PREC = {torch.float64: _lib.SHT_PREC_F64, torch.float32: _lib.SHT_PREC_F32}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(dtype, *tensors):
    if dtype not in _PREC:
        raise ValueError(f"the RHS kernels run in float32 or float64, got {dtype}")
    for t in tensors:
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            raise ValueError("every operand must be a CUDA tensor")
        if t.dtype != dtype:
            raise ValueError(f"mixed dtypes: {t.dtype} where {dtype} was expected")


def _c(t):
    return t.contiguous()


def momentum_bernoulli(vorticity, coriolis, u, v, wu, wv, virtual_temperature,
                       pressure_gradient, grad_lnps_east, grad_lnps_north, geopotential,
                       gas_constant):
    """``(momentum_u, momentum_v, bernoulli)``: the RHS momentum-forcing pair
    and Bernoulli function.  3-D operands ``(nlev, nlat, nlon)``; coriolis
    and the ln ps gradient ``(nlat, nlon)``."""
    dt = vorticity.dtype
    three = [vorticity, u, v, wu, wv, virtual_temperature, pressure_gradient, geopotential]
    two = [coriolis, grad_lnps_east, grad_lnps_north]
    _check(dt, *three, *two)
    shape = tuple(vorticity.shape)
    if len(shape) != 3 or any(tuple(t.shape) != shape for t in three):
        raise ValueError(f"the level fields must all be (nlev, nlat, nlon) = {shape}")
    if any(tuple(t.shape) != shape[1:] for t in two):
        raise ValueError(f"coriolis and the ln ps gradient must be (nlat, nlon) = {shape[1:]}")
    a = [_c(t) for t in (vorticity, coriolis, u, v, wu, wv, virtual_temperature,
                         pressure_gradient, grad_lnps_east, grad_lnps_north, geopotential)]
    out = [torch.empty(shape, dtype=dt, device=vorticity.device) for _ in range(3)]
    _lib.call("sht_rhs_momentum_bernoulli", _PREC[dt], shape[0], shape[1] * shape[2],
              *[_ptr(t) for t in a], float(gas_constant), *[_ptr(t) for t in out], _stream())
    return tuple(out)


def _blocks(scalar, block_shape):
    shape = tuple(scalar.shape)
    if len(shape) < 3 or shape[-3:] != tuple(block_shape):
        raise ValueError(f"the scalar is {shape} where (..., {', '.join(map(str, block_shape))}) "
                         "was expected")
    b = 1
    for d in shape[:-3]:
        b *= d
    return b


def tracer_flux(dp, scalar, u, v, out=None):
    """The horizontal mass-flux pair ``(dp*s*u, dp*s*v)``, contiguous as
    ``(2, *scalar.shape)`` (or written into ``out`` of that shape)."""
    dt = scalar.dtype
    _check(dt, dp, scalar, u, v)
    shape = tuple(dp.shape)
    if len(shape) != 3 or tuple(u.shape) != shape or tuple(v.shape) != shape:
        raise ValueError(f"dp, u and v must all be (nlev, nlat, nlon) = {shape}")
    blocks = _blocks(scalar, shape)
    if out is None:
        out = torch.empty((2, *scalar.shape), dtype=dt, device=scalar.device)
    elif tuple(out.shape) != (2, *scalar.shape) or not out.is_contiguous():
        raise ValueError("out must be a contiguous (2, *scalar.shape) tensor")
    _lib.call("sht_rhs_tracer_flux", _PREC[dt], blocks, shape[0], shape[1] * shape[2],
              _ptr(_c(dp)), _ptr(_c(scalar)), _ptr(_c(u)), _ptr(_c(v)), _ptr(out[0]),
              _ptr(out[1]), _stream())
    return out


def scalar_tendency(horizontal, vertical, scalar, dp_t, dp):
    """The flux-form scalar tendency ``(-h - vert - s*dp_t) / dp``."""
    dt = scalar.dtype
    _check(dt, horizontal, vertical, scalar, dp_t, dp)
    shape = tuple(dp.shape)
    if len(shape) != 3 or tuple(dp_t.shape) != shape:
        raise ValueError(f"dp and dp_t must both be (nlev, nlat, nlon) = {shape}")
    if tuple(horizontal.shape) != tuple(scalar.shape) or tuple(vertical.shape) != tuple(scalar.shape):
        raise ValueError("horizontal, vertical and scalar must share one shape")
    blocks = _blocks(scalar, shape)
    out = torch.empty(scalar.shape, dtype=dt, device=scalar.device)
    _lib.call("sht_rhs_scalar_tendency", _PREC[dt], blocks, shape[0], shape[1] * shape[2],
              _ptr(_c(horizontal)), _ptr(_c(vertical)), _ptr(_c(scalar)), _ptr(_c(dp_t)),
              _ptr(_c(dp)), _ptr(out), _stream())
    return out


def vertical_flux_divergence(scalar, omega_half, p_full, p_half):
    """The van Leer limited vertical flux divergence of ``scalar``
    ``(..., nlev, nlat, nlon)`` in the interface pressure velocity
    ``omega_half`` ``(nlev+1, nlat, nlon)``."""
    dt = scalar.dtype
    _check(dt, scalar, omega_half, p_full, p_half)
    shape = tuple(p_full.shape)
    if len(shape) != 3:
        raise ValueError("p_full must be (nlev, nlat, nlon)")
    half = (shape[0] + 1, shape[1], shape[2])
    if tuple(omega_half.shape) != half or tuple(p_half.shape) != half:
        raise ValueError(f"omega_half and p_half must be (nlev + 1, nlat, nlon) = {half}")
    blocks = _blocks(scalar, shape)
    out = torch.empty(scalar.shape, dtype=dt, device=scalar.device)
    _lib.call("sht_rhs_vertical_flux_divergence", _PREC[dt], blocks, shape[0],
              shape[1] * shape[2], _ptr(_c(scalar)), _ptr(_c(omega_half)), _ptr(_c(p_full)),
              _ptr(_c(p_half)), _ptr(out), _stream())
    return out
