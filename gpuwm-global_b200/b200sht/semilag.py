"""Semi-Lagrangian interpolation at departure points, on the GPU.

Mirrors the reference's ``arwen_global.semilag.tables.SphericalGridTables``
and ``arwen_global.semilag.interpolate`` (``Stencil``, ``zero_stencil``,
``gather_batch``, ``gather``, ``gather_linear_batch``; semilag/tables.py:98-258,
semilag/interpolate.py:87-500) with the same argument meaning and the same
``ValueError`` wording; the interpolation runs in ``libb200sht.so``
(``sht_sl_gather``, ``sht_sl_gather_linear``).  Arrays are CUDA tensors:
fields and departure coordinates ``(nlev, nlat, nlon)`` in the tables'
dtype (float32 or float64).  The whole-grid form only: a latitude-band
window (the reference's ``BandWindow``) is not part of this engine, whose
B200 holds every level and row of a T511 state at once.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any, Sequence

import numpy as np
import torch

from . import _lib

#: Fields per launch (interpolate.py DEFAULT_BATCH).
DEFAULT_BATCH = 16
#: Horizontal stencil widths: four-point cubic and six-point quintic.
ORDERS = (4, 6)
#: Limiter shapes: [cell min, cell max] and none.
LIMITERS = ("quasi_monotone", "none")

_DTYPES = {torch.float64: _lib.SHT_PREC_F64, torch.float32: _lib.SHT_PREC_F32}


def _torch_dtype(dtype) -> torch.dtype:
    if isinstance(dtype, torch.dtype):
        return dtype
    kind = np.dtype(dtype)
    if kind == np.float64:
        return torch.float64
    if kind == np.float32:
        return torch.float32
    raise ValueError(
        f"the semi-Lagrangian gather is compiled for float32 and float64 only, got {kind}")


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


class SphericalGridTables:
    """Device-resident gather geometry of one Gaussian grid and one dtype."""

    def __init__(self, handle, nlat: int, nlon: int, radius_m: float, dtype: torch.dtype,
                 device: torch.device):
        self._handle = handle
        self.nlat = nlat
        self.nlon = nlon
        self.radius_m = radius_m
        self.dtype = dtype
        self.device = device
        self.dlam = 2.0 * np.pi / nlon
        self.inv_dlam = 1.0 / self.dlam

    @classmethod
    def create(cls, grid, *, dtype=torch.float64, device=None) -> "SphericalGridTables":
        """Build the tables of ``grid`` (anything with ``nlat``, ``nlon``,
        ``lat_rad`` ascending and ``lon_rad``) on ``device``."""
        nlat, nlon = int(grid.nlat), int(grid.nlon)
        tdtype = _torch_dtype(dtype)
        lat = np.ascontiguousarray(np.asarray(grid.lat_rad, dtype=np.float64))
        if lat.shape != (nlat,):
            raise ValueError(f"lat_rad must have shape ({nlat},)")
        lon = np.ascontiguousarray(np.asarray(grid.lon_rad, dtype=np.float64))
        dev = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        handle = ctypes.c_void_p()
        dp = ctypes.POINTER(ctypes.c_double)
        with torch.cuda.device(dev):
            _lib.call("sht_sl_tables_create", nlat, nlon, lat.ctypes.data_as(dp),
                      lon.ctypes.data_as(dp) if lon.shape == (nlon,) else None,
                      _DTYPES[tdtype], ctypes.byref(handle))
        return cls(handle, nlat, nlon, float(getattr(grid, "radius_m", 6371220.0)), tdtype, dev)

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value and _lib._lib is not None:
            _lib._lib.sht_sl_tables_destroy(handle)
            self._handle = None

    @property
    def shape(self) -> tuple[int, int]:
        return self.nlat, self.nlon

    def equatorial_spacing_m(self) -> float:
        """``a * 2*pi / nlon``: one zonal cell at the equator."""
        return self.radius_m * self.dlam

    def host_tables(self, order: int = 4) -> dict:
        """float64 host copies of one width's tables (for checks)."""
        rows, bins = ctypes.c_int(), ctypes.c_int()
        scale = ctypes.c_double()
        _lib.call("sht_sl_tables_read", self._handle, int(order), None, None, None, None, None,
                  ctypes.byref(rows), ctypes.byref(bins), ctypes.byref(scale))
        r, b = rows.value, bins.value
        out = {"lat_ext": np.empty(r), "mrden": np.empty((self.nlat + 1, int(order))),
               "mlut": np.empty(b, np.int32), "rowoff": np.empty(r, np.int32),
               "rowshift": np.empty(r, np.int32)}
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        _lib.call("sht_sl_tables_read", self._handle, int(order),
                  out["lat_ext"].ctypes.data_as(dp), out["mrden"].ctypes.data_as(dp),
                  out["mlut"].ctypes.data_as(ip), out["rowoff"].ctypes.data_as(ip),
                  out["rowshift"].ctypes.data_as(ip), None, None, None)
        out["lookup_bins"], out["lut_scale"] = b, scale.value
        return out


@dataclass(frozen=True)
class Stencil:
    """Departure coordinates of every arrival point of one grid: ``xi`` in
    continuous zonal index, ``phi`` in radians, ``level`` in continuous
    full-level index, each ``(nlev, nlat, nlon)``."""

    xi: Any
    phi: Any
    level: Any
    tables: SphericalGridTables

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(int(s) for s in self.xi.shape)  # type: ignore[return-value]

    @property
    def source_shape(self) -> tuple[int, int, int]:
        return self.shape

    def __post_init__(self) -> None:
        shape = tuple(int(s) for s in self.xi.shape)
        if len(shape) != 3:
            raise ValueError(f"departure coordinates must be (nlev, nlat, nlon), got {shape}")
        if shape[1:] != self.tables.shape:
            raise ValueError(
                f"departure coordinates are {shape[1:]} where {self.tables.shape} were "
                f"expected on a {self.tables.shape} grid")
        if shape[0] < 4:
            raise ValueError(f"a four-point vertical stencil needs nlev >= 4, got {shape[0]}")
        for name in ("phi", "level"):
            other = tuple(int(s) for s in getattr(self, name).shape)
            if other != shape:
                raise ValueError(f"{name} is {other} where xi is {shape}")
        for name in ("xi", "phi", "level"):
            t = getattr(self, name)
            if not (isinstance(t, torch.Tensor) and t.is_cuda):
                raise ValueError(f"{name} must be a CUDA tensor")
            if t.dtype != self.tables.dtype:
                raise ValueError(f"{name} is {t.dtype} where the grid tables were built for "
                                 f"{self.tables.dtype}")
            if not t.is_contiguous():
                object.__setattr__(self, name, t.contiguous())


def zero_stencil(tables: SphericalGridTables, nlev: int) -> Stencil:
    """The identity stencil: every arrival point departs from itself."""
    nlat, nlon = tables.shape
    host = tables.host_tables(4)
    dev, dt = tables.device, tables.dtype
    lat = torch.as_tensor(host["lat_ext"][2:nlat + 2], dtype=dt, device=dev)
    xi = torch.arange(nlon, dtype=dt, device=dev)[None, None, :].expand(nlev, nlat, nlon)
    phi = lat[None, :, None].expand(nlev, nlat, nlon)
    lev = torch.arange(nlev, dtype=dt, device=dev)[:, None, None].expand(nlev, nlat, nlon)
    return Stencil(xi=xi.contiguous(), phi=phi.contiguous(), level=lev.contiguous(),
                   tables=tables)


def _limiter_of(monotone) -> str:
    if isinstance(monotone, str):
        return monotone
    return "quasi_monotone" if monotone else "none"


def _validate(limiter: str, deficit: bool, order: int) -> None:
    if limiter not in LIMITERS:
        raise ValueError("the semi-Lagrangian gather's limiter must be one of "
                         + ", ".join(repr(item) for item in LIMITERS) + f", got {limiter!r}")
    if int(order) not in ORDERS:
        raise ValueError("the semi-Lagrangian gather's horizontal order must be one of "
                         + ", ".join(str(item) for item in ORDERS) + f", got {order!r}")
    if limiter == "none" and deficit:
        raise ValueError(
            "the clip deficit is the mass the limiter moved, so an unlimited gather has none "
            "to report; ask for a limiter or do not ask for the deficit")
    if deficit and int(order) != 4:
        raise ValueError(
            "the clip deficit is reported by the cubic gather only: the additive mass fixer "
            "reads it for the limited species, which ride the cubic stencil, and a quintic "
            "deficit would be a number nothing consumes")


def _check_fields(fields, stencil: Stencil) -> None:
    shape = stencil.source_shape
    for index, field in enumerate(fields):
        got = tuple(int(s) for s in field.shape)
        if got != shape:
            raise ValueError(f"field {index} is {got} where the stencil reads {shape}")
        if field.dtype != stencil.tables.dtype:
            raise ValueError(
                f"field {index} is {field.dtype} where the grid tables were built for "
                f"{stencil.tables.dtype}; a mixed-precision gather would read the wrong bytes, "
                f"not the wrong answer")
        if not field.is_cuda:
            raise ValueError(f"field {index} must be a CUDA tensor")


def _source_block(chunk):
    """The batch's fields as one contiguous (count, nlev, nlat, nlon) block;
    a single contiguous field is used in place."""
    if len(chunk) == 1 and chunk[0].is_contiguous():
        return chunk[0][None]
    return torch.stack(list(chunk), dim=0).contiguous()


def gather_batch(fields: Sequence[torch.Tensor], stencil: Stencil, *, monotone: Any = True,
                 batch: int = DEFAULT_BATCH, deficit: bool = False, order: int = 4) -> list:
    """Read every field at the stencil's departure points (tricubic for
    ``order = 4``, quintic horizontal for 6).  ``deficit=True`` (with a
    limiter) returns ``(value, clip_deficit)`` pairs."""
    if not fields:
        return []
    _check_fields(fields, stencil)
    if int(batch) < 1:
        raise ValueError("batch must be >= 1")
    limiter = _limiter_of(monotone)
    order = int(order)
    _validate(limiter, deficit, order)
    if order == 6 and stencil.tables.nlat < 6:
        raise ValueError(
            f"the quintic gather needs six meridional rows and this grid has "
            f"{stencil.tables.nlat}; the six-point tables were not built")
    nlev = stencil.shape[0]
    lim = _lib.SHT_SL_QUASI_MONOTONE if limiter == "quasi_monotone" else _lib.SHT_SL_NONE
    out: list = []
    for start in range(0, len(fields), int(batch)):
        chunk = fields[start:start + int(batch)]
        src = _source_block(chunk)
        count = len(chunk)
        dst = torch.empty((count, *stencil.shape), dtype=src.dtype, device=src.device)
        cut = torch.empty_like(dst) if deficit else None
        _lib.call("sht_sl_gather", stencil.tables._handle, order, lim, 1 if deficit else 0,
                  _ptr(src), count, nlev, _ptr(stencil.xi), _ptr(stencil.phi),
                  _ptr(stencil.level), _ptr(dst), _ptr(cut) if cut is not None else None,
                  _stream())
        if deficit:
            out.extend((dst[i], cut[i]) for i in range(count))
        else:
            out.extend(dst[i] for i in range(count))
    return out


def gather(field: torch.Tensor, stencil: Stencil, *, monotone: Any = True, order: int = 4):
    """One field at the stencil's departure points."""
    return gather_batch([field], stencil, monotone=monotone, order=order)[0]


def gather_linear_batch(fields: Sequence[torch.Tensor], stencil: Stencil, *,
                        batch: int = DEFAULT_BATCH) -> list:
    """Every field read trilinearly inside the cubic gather's limiter cell."""
    if not fields:
        return []
    _check_fields(fields, stencil)
    if int(batch) < 1:
        raise ValueError("batch must be >= 1")
    nlev = stencil.shape[0]
    out: list = []
    for start in range(0, len(fields), int(batch)):
        chunk = fields[start:start + int(batch)]
        src = _source_block(chunk)
        count = len(chunk)
        dst = torch.empty((count, *stencil.shape), dtype=src.dtype, device=src.device)
        _lib.call("sht_sl_gather_linear", stencil.tables._handle, _ptr(src), count, nlev,
                  _ptr(stencil.xi), _ptr(stencil.phi), _ptr(stencil.level), _ptr(dst),
                  _stream())
        out.extend(dst[i] for i in range(count))
    return out
