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
marching down the levels.  The reference's calling form
``momentum_bernoulli_kernel(xp)(...)`` (and the other three) is kept: each
factory returns a callable with the kernel's operand order, outputs
optional.
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
                       gas_constant, out=None):
    """``(momentum_u, momentum_v, bernoulli)``: the RHS momentum-forcing pair
    and Bernoulli function.  3-D operands ``(nlev, nlat, nlon)``; coriolis
    and the ln ps gradient ``(nlat, nlon)``; ``out``: three contiguous
    tensors to write instead of new ones."""
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
    out = _outputs(out, 3, shape, dt, vorticity.device)
    _lib.call("sht_rhs_momentum_bernoulli", _PREC[dt], shape[0], shape[1] * shape[2],
              *[_ptr(t) for t in a], float(gas_constant), *[_ptr(t) for t in out], _stream())
    return tuple(out)


def _outputs(out, count, shape, dtype, device):
    if out is None:
        return [torch.empty(shape, dtype=dtype, device=device) for _ in range(count)]
    out = list(out)
    if len(out) != count:
        raise ValueError(f"out must hold {count} tensors")
    for t in out:
        if (not isinstance(t, torch.Tensor) or tuple(t.shape) != tuple(shape) or t.dtype != dtype
                or t.device != device or not t.is_contiguous()):
            raise ValueError(f"every output must be a contiguous {dtype} CUDA tensor of shape "
                             f"{tuple(shape)}")
    return out


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
    if out is None:
        out = torch.empty((2, *scalar.shape), dtype=dt, device=scalar.device)
    elif tuple(out.shape) != (2, *scalar.shape) or not out.is_contiguous():
        raise ValueError("out must be a contiguous (2, *scalar.shape) tensor")
    _tracer_flux_into(dp, scalar, u, v, out[0], out[1])
    return out


def _tracer_flux_into(dp, scalar, u, v, fx, fy):
    dt = scalar.dtype
    _check(dt, dp, scalar, u, v)
    shape = tuple(dp.shape)
    if len(shape) != 3 or tuple(u.shape) != shape or tuple(v.shape) != shape:
        raise ValueError(f"dp, u and v must all be (nlev, nlat, nlon) = {shape}")
    blocks = _blocks(scalar, shape)
    fx, fy = _outputs((fx, fy), 2, tuple(scalar.shape), dt, scalar.device)
    _lib.call("sht_rhs_tracer_flux", _PREC[dt], blocks, shape[0], shape[1] * shape[2],
              _ptr(_c(dp)), _ptr(_c(scalar)), _ptr(_c(u)), _ptr(_c(v)), _ptr(fx), _ptr(fy),
              _stream())
    return fx, fy


def scalar_tendency(horizontal, vertical, scalar, dp_t, dp, out=None):
    """The flux-form scalar tendency ``(-h - vert - s*dp_t) / dp``."""
    dt = scalar.dtype
    _check(dt, horizontal, vertical, scalar, dp_t, dp)
    shape = tuple(dp.shape)
    if len(shape) != 3 or tuple(dp_t.shape) != shape:
        raise ValueError(f"dp and dp_t must both be (nlev, nlat, nlon) = {shape}")
    if tuple(horizontal.shape) != tuple(scalar.shape) or tuple(vertical.shape) != tuple(scalar.shape):
        raise ValueError("horizontal, vertical and scalar must share one shape")
    blocks = _blocks(scalar, shape)
    (out,) = _outputs(None if out is None else (out,), 1, tuple(scalar.shape), dt,
                      scalar.device)
    _lib.call("sht_rhs_scalar_tendency", _PREC[dt], blocks, shape[0], shape[1] * shape[2],
              _ptr(_c(horizontal)), _ptr(_c(vertical)), _ptr(_c(scalar)), _ptr(_c(dp_t)),
              _ptr(_c(dp)), _ptr(out), _stream())
    return out


def vertical_flux_divergence(scalar, omega_half, p_full, p_half, out=None):
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
    (out,) = _outputs(None if out is None else (out,), 1, tuple(scalar.shape), dt,
                      scalar.device)
    _lib.call("sht_rhs_vertical_flux_divergence", _PREC[dt], blocks, shape[0],
              shape[1] * shape[2], _ptr(_c(scalar)), _ptr(_c(omega_half)), _ptr(_c(p_full)),
              _ptr(_c(p_half)), _ptr(out), _stream())
    return out


# ------------------------------------------- the reference's kernel factories
def momentum_bernoulli_kernel(xp=None):
    """The reference's ``momentum_bernoulli_kernel(xp)`` (fused.py:233-261):
    a callable taking the kernel's operands in its order ``(zeta, cor, u, v,
    wu, wv, tv, pg, ge, gn, phi, rgas[, mu, mv, bern])`` and returning
    ``(mu, mv, bern)``, written into the given outputs when they are passed.
    ``xp`` is accepted for the reference's signature."""
    def run(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, rgas, mu=None, mv=None, bern=None):
        outs = None if mu is None else (mu, mv, bern)
        return momentum_bernoulli(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, float(rgas),
                                  out=outs)
    return run


def tracer_flux_kernel(xp=None):
    """The reference's ``tracer_flux_kernel(xp)`` (fused.py:264-281):
    ``(dp, s, u, v[, fx, fy]) -> (fx, fy)``, ``s`` with any leading tracer
    axes ahead of ``dp``'s ``(nlev, nlat, nlon)``."""
    def run(dp, s, u, v, fx=None, fy=None):
        if fx is None:
            fx = torch.empty(s.shape, dtype=s.dtype, device=s.device)
            fy = torch.empty_like(fx)
        return _tracer_flux_into(dp, s, u, v, fx, fy)
    return run


def scalar_tendency_kernel(xp=None):
    """The reference's ``scalar_tendency_kernel(xp)`` (fused.py:284-295):
    ``(h, vert, s, dpt, dp[, out]) -> (-h - vert - s*dpt) / dp``."""
    def run(h, vert, s, dpt, dp, out=None):
        return scalar_tendency(h, vert, s, dpt, dp, out=out)
    return run


def vertical_flux_divergence_kernel(xp=None):
    """The reference's ``vertical_flux_divergence_kernel(xp)``
    (fused.py:366-386): ``(s, w, pf, ph, nlev, horiz[, out])``, ``nlev`` and
    ``horiz`` checked against the shapes."""
    def run(s, w, pf, ph, nlev, horiz, out=None):
        if int(nlev) != int(pf.shape[0]) or int(horiz) != int(pf.shape[1] * pf.shape[2]):
            raise ValueError(f"nlev={nlev}, horiz={horiz} do not match p_full's shape "
                             f"{tuple(pf.shape)}")
        return vertical_flux_divergence(s, w, pf, ph, out=out)
    return run
