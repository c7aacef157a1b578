"""Semi-Lagrangian interpolation at departure points, on the GPU.

Mirrors the reference's ``arwen_global.semilag.tables.SphericalGridTables``,
``arwen_global.semilag.interpolate`` (``Stencil``, ``zero_stencil``,
``gather_batch``, ``gather``, ``gather_linear_batch``; semilag/tables.py:98-258,
semilag/interpolate.py:87-500) and the fixed-point departure search of
``arwen_global.semilag.trajectory`` (``CartesianWind``, ``cartesian_wind``,
``local_wind``, ``departure_points``, ``TrajectoryDiagnostics``) with the same
argument meaning and the same ``ValueError`` wording; the interpolation and
the search run in ``libb200sht.so`` (``sht_sl_gather``,
``sht_sl_gather_linear``, ``sht_sl_departure``).  Arrays are CUDA tensors:
fields and departure coordinates ``(nlev, nlat, nlon)`` in the tables'
dtype (float32 or float64).  Latitude-band windows (the reference's
``BandWindow``, ``HaloEscape``, ``SphericalGridTables.window``) give the
banded step's gathers and searches over a band's rows from fields that hold
the band and its halo (``sht_sl_gather_band``, ``sht_sl_departure_band``).
The search's gate is the reference's too (trajectory.py:121-155, 755-1560):
``lipschitz`` (the flow deformation, one kernel: ``sht_sl_lipschitz``),
``LipschitzDiagnostics``, ``refuse_trajectory_fold``, ``convergence``,
``converged_departure_points`` and ``level_rate_from_mass_flux``.
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

    def window(self, source: slice, arrival: slice) -> "BandWindow":
        """The tables of one latitude band read through its row halo
        (cached per (held rows, band rows))."""
        key = (int(source.start), int(source.stop), int(arrival.start), int(arrival.stop))
        cache = self.__dict__.setdefault("_windows", {})
        win = cache.get(key)
        if win is None:
            win = cache[key] = BandWindow.create(self, source, arrival)
        return win

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


class HaloEscape(ValueError):
    """A departure point, or a trajectory iterate, read a latitude row the
    band does not hold (the reference's tables.HaloEscape)."""

    def __init__(self, window: "BandWindow", what: str):
        self.window = window
        super().__init__(
            f"the semi-Lagrangian {what} of latitude rows {window.arrival.start}.."
            f"{window.arrival.stop} read a row outside the rows {window.source.start}.."
            f"{window.source.stop} the band holds: a departure point left the band's row "
            "halo, and reading on would return a value from a row the band does not have")


class BandWindow:
    """One latitude band of the semi-Lagrangian step (``arrival`` rows) and
    the rows its fields hold (``source``, the band plus a row halo).

    A window has one escape flag on the device.  Its band calls (each a
    ``clear_escape`` .. kernels .. ``raise_if_escaped`` sequence) must run on
    one stream, one after another: two calls of the same window in flight on
    different streams would lower and read each other's flag.  The reference's
    band windows share the same rule."""

    def __init__(self, tables, source: slice, arrival: slice, handle):
        self.tables = tables
        self.source = source
        self.arrival = arrival
        self._handle = handle

    @classmethod
    def create(cls, tables: SphericalGridTables, source: slice, arrival: slice) -> "BandWindow":
        s0, s1, a0, a1 = int(source.start), int(source.stop), int(arrival.start), int(arrival.stop)
        handle = ctypes.c_void_p()
        with torch.cuda.device(tables.device):
            _lib.call("sht_sl_window_create", tables._handle, s0, s1, a0, a1, ctypes.byref(handle))
        return cls(tables, slice(s0, s1), slice(a0, a1), handle)

    def __del__(self):
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value and _lib._lib is not None:
            _lib._lib.sht_sl_window_destroy(handle)
            self._handle = None

    def clear_escape(self) -> None:
        """Lower the escape flag before a band's kernels run."""
        _lib.call("sht_sl_window_escape", self._handle, 1, None, _stream())

    def raise_if_escaped(self, what: str) -> None:
        """Refuse by name if a band kernel since clear_escape read a row the
        band does not hold (one device read, which waits for the stream)."""
        flag = ctypes.c_int(0)
        _lib.call("sht_sl_window_escape", self._handle, 0, ctypes.byref(flag), _stream())
        if flag.value:
            raise HaloEscape(self, what)

    @property
    def source_rows(self) -> int:
        return int(self.source.stop - self.source.start)

    @property
    def arrival_rows(self) -> int:
        return int(self.arrival.stop - self.arrival.start)

    @property
    def lead(self) -> int:
        """The band's first row's index inside the held rows."""
        return int(self.arrival.start - self.source.start)

    @property
    def local(self) -> slice:
        """The band's rows as a slice of the held rows."""
        return slice(self.lead, self.lead + self.arrival_rows)

    def arrival_shape(self, nlev: int) -> tuple[int, int, int]:
        return int(nlev), self.arrival_rows, int(self.tables.nlon)

    def source_shape(self, nlev: int) -> tuple[int, int, int]:
        return int(nlev), self.source_rows, int(self.tables.nlon)


@dataclass(frozen=True)
class Stencil:
    """Departure coordinates of every arrival point of one grid: ``xi`` in
    continuous zonal index, ``phi`` in radians, ``level`` in continuous
    full-level index, each ``(nlev, nlat, nlon)``."""

    xi: Any
    phi: Any
    level: Any
    tables: SphericalGridTables
    #: The latitude band these arrival points are and the rows its source
    #: fields hold, or None for the whole grid.
    window: "BandWindow | None" = None

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(int(s) for s in self.xi.shape)  # type: ignore[return-value]

    @property
    def source_shape(self) -> tuple[int, int, int]:
        if self.window is None:
            return self.shape
        return self.window.source_shape(self.shape[0])

    def __post_init__(self) -> None:
        shape = tuple(int(s) for s in self.xi.shape)
        if len(shape) != 3:
            raise ValueError(f"departure coordinates must be (nlev, nlat, nlon), got {shape}")
        expected = (self.tables.shape if self.window is None
                    else (self.window.arrival_rows, self.tables.nlon))
        if shape[1:] != expected:
            raise ValueError(
                f"departure coordinates are {shape[1:]} where {expected} were "
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
                 batch: int = DEFAULT_BATCH, deficit: bool = False, order: int = 4,
                 defer_escape: bool = False) -> list:
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
    window = stencil.window
    if window is not None and not defer_escape:
        window.clear_escape()
    out: list = []
    for start in range(0, len(fields), int(batch)):
        chunk = fields[start:start + int(batch)]
        src = _source_block(chunk)
        count = len(chunk)
        dst = torch.empty((count, *stencil.shape), dtype=src.dtype, device=src.device)
        cut = torch.empty_like(dst) if deficit else None
        name, handle = (("sht_sl_gather", stencil.tables._handle) if window is None
                        else ("sht_sl_gather_band", window._handle))
        _lib.call(name, handle, order, lim, 1 if deficit else 0,
                  _ptr(src), count, nlev, _ptr(stencil.xi), _ptr(stencil.phi),
                  _ptr(stencil.level), _ptr(dst), _ptr(cut) if cut is not None else None,
                  _stream())
        if deficit:
            out.extend((dst[i], cut[i]) for i in range(count))
        else:
            out.extend(dst[i] for i in range(count))
    if window is not None and not defer_escape:
        window.raise_if_escaped("gather")
    return out


def gather(field: torch.Tensor, stencil: Stencil, *, monotone: Any = True, order: int = 4):
    """One field at the stencil's departure points."""
    return gather_batch([field], stencil, monotone=monotone, order=order)[0]


def gather_linear_batch(fields: Sequence[torch.Tensor], stencil: Stencil, *,
                        batch: int = DEFAULT_BATCH) -> list:
    """Every field read trilinearly inside the cubic gather's limiter cell."""
    if not fields:
        return []
    if stencil.window is not None:
        raise ValueError(
            "the trilinear gather reads the whole grid's rows; assemble the whole stencil "
            "before asking for it")
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


# --------------------------------------------------------------- trajectory
# The reference's semilag/trajectory.py: CartesianWind, cartesian_wind,
# local_wind, TrajectoryDiagnostics, meridional_grid_length_m and
# departure_points (trajectory.py:50-120, 158-358, 440-490).

#: Solvers of the departure-point equation: the fixed-point pass (the
#: reference's default and its numpy specification), Newton's method on the
#: same equation, and Newton with a backtracking line search on the residual
#: (the form that converges where (dt/2)|J| nears one).
TRAJECTORY_SOLVERS = ("fixed_point", "newton", "newton_ls")


@dataclass(frozen=True)
class CartesianWind:
    """Geocentric Cartesian components of the horizontal wind (m/s) and the
    vertical velocity in level indices per second, at full levels."""

    vx: Any
    vy: Any
    vz: Any
    level_rate: Any

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(int(s) for s in self.vx.shape)  # type: ignore[return-value]

    def arrays(self) -> tuple:
        return (self.vx, self.vy, self.vz, self.level_rate)


def _trig(tables: SphericalGridTables):
    nlat, nlon = tables.shape
    host = tables.host_tables(4)
    dev, dt = tables.device, tables.dtype
    lat = torch.as_tensor(host["lat_ext"][2:nlat + 2], dtype=dt, device=dev)
    lon = torch.as_tensor(np.arange(nlon) * tables.dlam, dtype=dt, device=dev)
    return (torch.sin(lat)[None, :, None], torch.cos(lat)[None, :, None],
            torch.sin(lon)[None, None, :], torch.cos(lon)[None, None, :])


def cartesian_wind(u, v, tables: SphericalGridTables):
    """Local east-north wind as geocentric Cartesian components."""
    sph, cph, sla, cla = _trig(tables)
    vx = -u * sla - v * sph * cla
    vy = u * cla - v * sph * sla
    vz = v * cph + torch.zeros_like(u)
    return vx, vy, vz


def local_wind(vx, vy, vz, tables: SphericalGridTables):
    """Geocentric Cartesian components back to the local east-north wind."""
    sph, cph, sla, cla = _trig(tables)
    u = -vx * sla + vy * cla
    v = -vx * sph * cla - vy * sph * sla + vz * cph
    return u, v


@dataclass(frozen=True)
class TrajectoryDiagnostics:
    iterations: int
    dt_s: float
    #: largest last-iteration move, metres, and in meridional grid lengths
    move_max_m: float
    move_max_cells: float
    #: largest last-iteration move of the level coordinate
    move_max_levels: float
    #: largest displacement of the finished trajectory
    displacement_max_m: float
    displacement_max_cells: float
    displacement_max_levels: float

    def as_dict(self) -> dict:
        return {
            "semilag_trajectory_iterations": self.iterations,
            "semilag_trajectory_dt_s": self.dt_s,
            "semilag_trajectory_move_max_m": self.move_max_m,
            "semilag_trajectory_move_max_cells": self.move_max_cells,
            "semilag_trajectory_move_max_levels": self.move_max_levels,
            "semilag_displacement_max_m": self.displacement_max_m,
            "semilag_displacement_max_cells": self.displacement_max_cells,
            "semilag_displacement_max_levels": self.displacement_max_levels,
        }


def meridional_grid_length_m(tables: SphericalGridTables) -> np.ndarray:
    """``a * dphi`` per latitude row (half the spread of the neighbouring
    rows, the pole rows through their reflections)."""
    lat_ext = tables.host_tables(4)["lat_ext"]
    nlat = tables.nlat
    return tables.radius_m * 0.5 * (lat_ext[3:nlat + 3] - lat_ext[1:nlat + 1])


def _diagnostics(stencil: Stencil, move_m, move_k, tables, dt_s, iterations):
    nlev, nrows, nlon = stencil.shape
    nlat = tables.nlat
    rows = slice(0, nlat) if stencil.window is None else stencil.window.arrival
    dt = tables.dtype
    dev = tables.device
    cell = torch.as_tensor(meridional_grid_length_m(tables)[rows], dtype=dt,
                           device=dev)[None, :, None]
    lat = torch.as_tensor(tables.host_tables(4)["lat_ext"][2:nlat + 2][rows], dtype=dt,
                          device=dev)[None, :, None]
    index = torch.arange(nlon, dtype=dt, device=dev)[None, None, :]
    lev0 = torch.arange(nlev, dtype=dt, device=dev)[:, None, None]
    # great-circle distance through the haversine (no floor from arccos)
    dphi = 0.5 * (stencil.phi - lat)
    dlon = 0.5 * (stencil.xi - index) * tables.dlam
    hav = torch.sin(dphi) ** 2 + torch.cos(lat) * torch.cos(stencil.phi) * torch.sin(dlon) ** 2
    dist = (2.0 * tables.radius_m) * torch.arcsin(torch.sqrt(torch.clamp(hav, 0.0, 1.0)))
    maxima = torch.stack([move_m.max(), (move_m / cell).max(), move_k.max(), dist.max(),
                          (dist / cell).max(), (stencil.level - lev0).abs().max()]).tolist()
    return TrajectoryDiagnostics(int(iterations), float(dt_s), *[float(x) for x in maxima])


_SOLVER_CALLS = {"fixed_point": "sht_sl_departure", "newton": "sht_sl_departure_newton",
                 "newton_ls": "sht_sl_departure_newton_ls"}


def search_into(tables: SphericalGridTables, fields: Sequence[torch.Tensor], iterations: int,
                dt_s: float, outs: Sequence[torch.Tensor], solver: str = "fixed_point") -> None:
    """The search kernel alone: ``fields`` = (vx, vy, vz, level_rate) of the
    advecting wind then of the extrapolated one, contiguous; ``outs`` = xi,
    phi, level, move_m, move_k.  No checks beyond the library's."""
    nlev = int(fields[0].shape[0])
    name = _SOLVER_CALLS[solver]
    _lib.call(name, tables._handle, nlev, *[_ptr(t) for t in fields],
              int(iterations), float(dt_s), float(tables.radius_m), *[_ptr(t) for t in outs],
              _stream())


def departure_points(wind: CartesianWind, tables: SphericalGridTables, dt_s: float, *,
                     iterations: int = 3, extrapolated: CartesianWind | None = None,
                     window: BandWindow | None = None, defer_escape: bool = False,
                     solver: str = "fixed_point") -> tuple[Stencil, TrajectoryDiagnostics]:
    """The departure point of every arrival point of the grid (all
    iterations in one launch).  With a ``window`` the arrival points are the
    band's rows: ``wind`` holds the band and its halo, ``extrapolated`` the
    band's own rows (by default those rows of ``wind``); a search that reads
    a row the band does not hold is refused by name (HaloEscape)."""
    shape = wind.shape
    nlev, nrows, nlon = shape
    held = tables.nlat if window is None else window.source_rows
    if (nrows, nlon) != (held, tables.nlon):
        raise ValueError(f"the wind is {(nrows, nlon)} where {(held, tables.nlon)} rows were "
                         f"expected on a {tables.shape} grid")
    if nlev < 4:
        raise ValueError(f"nlev >= 4 is required, got {nlev}")
    if int(iterations) < 1:
        raise ValueError(
            "the departure-point search needs at least one iteration; zero would ship the "
            "explicit first guess, which is first order in dt and is not a trajectory")
    if solver not in TRAJECTORY_SOLVERS:
        raise ValueError(f"trajectory solver must be one of {TRAJECTORY_SOLVERS}, got {solver!r}")
    out_shape = shape if window is None else window.arrival_shape(nlev)
    ex = wind if extrapolated is None else extrapolated
    if window is not None and extrapolated is None:
        ex = CartesianWind(*(f[:, window.local].contiguous() for f in wind.arrays()))
    for name, arr, want in (("wind", wind, shape), ("extrapolated", ex, out_shape)):
        for field in arr.arrays():
            if tuple(int(s) for s in field.shape) != want:
                raise ValueError(f"{name} fields must all be {want}")
            if field.dtype != tables.dtype:
                raise ValueError(f"{name} is {field.dtype} where the grid tables were built for "
                                 f"{tables.dtype}")
            if not field.is_cuda:
                raise ValueError(f"{name} fields must be CUDA tensors")
    ins = [f.contiguous() for f in wind.arrays()] + [f.contiguous() for f in ex.arrays()]
    outs = [torch.empty(out_shape, dtype=tables.dtype, device=ins[0].device) for _ in range(5)]
    if window is None:
        search_into(tables, ins, int(iterations), float(dt_s), outs, solver=solver)
    else:
        if not defer_escape:
            window.clear_escape()
        _lib.call("sht_sl_departure_band", window._handle, TRAJECTORY_SOLVERS.index(solver), nlev,
                  *[_ptr(t) for t in ins], int(iterations), float(dt_s), float(tables.radius_m),
                  *[_ptr(t) for t in outs], _stream())
        if not defer_escape:
            window.raise_if_escaped("departure-point search")
    xi, phi, lev, move_m, move_k = outs
    stencil = Stencil(xi=xi, phi=phi, level=lev, tables=tables, window=window)
    return stencil, _diagnostics(stencil, move_m, move_k, tables, dt_s, iterations)


# ------------------------------------------------------- trajectory gate
def level_rate_from_mass_flux(omega_half, *, p_full, xp=None):
    """The vertical rate in level indices per second at full levels
    (trajectory.py:121-155): the interface mass flux ``etadot dp/deta``
    (Pa/s, ``nlev + 1`` interfaces, zero at both boundaries) divided by the
    pressure distance between the neighbouring full levels, averaged onto
    the levels.  ``p_full`` is the full-level pressure, ``(nlev, ...)``
    broadcasting against the interfaces' trailing axes.  Works on torch
    tensors and numpy arrays alike (``xp`` is accepted for the reference's
    signature and not needed)."""
    nlev = int(p_full.shape[0])
    if int(omega_half.shape[0]) != nlev + 1:
        raise ValueError(f"omega_half must have {nlev + 1} interfaces for {nlev} layers, "
                         f"got {int(omega_half.shape[0])}")
    if isinstance(omega_half, torch.Tensor):
        s_half = torch.zeros_like(omega_half)
        p = torch.as_tensor(p_full, dtype=omega_half.dtype, device=omega_half.device)
    else:
        s_half = np.zeros_like(omega_half)
        p = p_full
    distance = p[1:] - p[:-1]  # broadcast against omega_half[1:nlev] as given
    s_half[1:nlev] = omega_half[1:nlev] / distance
    return 0.5 * (s_half[:nlev] + s_half[1:nlev + 1])


@dataclass(frozen=True)
class LipschitzDiagnostics:
    """The flow deformation: the fold determinants the trajectory gate reads
    and the Jacobian norms reported beside them (the reference's
    LipschitzDiagnostics, trajectory.py:755-952, same fields, properties
    and receipt keys).  ``fold_determinant`` = the smaller of
    min det(I - (dt/2) J_ex) (arrival side) and min det(I + (dt/2) J)
    (departure side); the norms are per second (``jacobian_*``) and times dt
    (``lipschitz_*``)."""

    dt_s: float
    reference_length_m: float
    lipschitz: float
    lipschitz_frobenius: float
    lipschitz_horizontal: float
    jacobian_spectral_s: float
    jacobian_frobenius_s: float
    jacobian_horizontal_s: float
    lipschitz_vertical: float = 0.0
    jacobian_vertical_s: float = 0.0
    lipschitz_mixed: float = 0.0
    lipschitz_balanced: float = 0.0
    jacobian_balanced_s: float = 0.0
    fold_determinant_arrival: float = 1.0
    fold_determinant_departure: float = 1.0
    fold_where_arrival: str = ""
    fold_where_departure: str = ""

    @property
    def fold_determinant(self) -> float:
        return min(self.fold_determinant_arrival, self.fold_determinant_departure)

    @property
    def fold_side(self) -> str:
        return ("arrival" if self.fold_determinant_arrival <= self.fold_determinant_departure
                else "departure")

    @property
    def binding_direction(self) -> str:
        if self.lipschitz_balanced > 1.000001 * max(self.lipschitz_horizontal,
                                                     self.lipschitz_vertical):
            return "coupling"
        return "vertical" if self.lipschitz_vertical > self.lipschitz_horizontal else "horizontal"

    def as_dict(self) -> dict:
        return {
            "semilag_lipschitz": self.lipschitz,
            "semilag_lipschitz_frobenius": self.lipschitz_frobenius,
            "semilag_lipschitz_horizontal": self.lipschitz_horizontal,
            "semilag_lipschitz_vertical": self.lipschitz_vertical,
            "semilag_lipschitz_balanced": self.lipschitz_balanced,
            "semilag_lipschitz_mixed": self.lipschitz_mixed,
            "semilag_jacobian_balanced_s": self.jacobian_balanced_s,
            "semilag_jacobian_spectral_s": self.jacobian_spectral_s,
            "semilag_jacobian_frobenius_s": self.jacobian_frobenius_s,
            "semilag_jacobian_horizontal_s": self.jacobian_horizontal_s,
            "semilag_jacobian_vertical_s": self.jacobian_vertical_s,
            "semilag_lipschitz_reference_length_m": self.reference_length_m,
            "semilag_lipschitz_dt_s": self.dt_s,
            "semilag_fold_determinant": self.fold_determinant,
            "semilag_fold_determinant_arrival": self.fold_determinant_arrival,
            "semilag_fold_determinant_departure": self.fold_determinant_departure,
        }


#: Levels per pass of the reference's diagnostic (accepted; the kernel here
#: takes every level in one pass and holds no volume-sized temporary).
LIPSCHITZ_LEVEL_CHUNK = 8
#: The most iterations the departure search takes on a retry (trajectory.py).
MAXIMUM_TRAJECTORY_ITERATIONS = 8
#: The default floor under the fold determinant (trajectory.py).
DEFAULT_MINIMUM_FOLD_DETERMINANT = 0.2


def _where(flat: int, shape, lat_ext, dlam, a0: int) -> str:
    _, nr, nl = shape
    kk, jj, ii = flat // (nr * nl), (flat // nl) % nr, flat % nl
    lat_d = float(np.degrees(lat_ext[jj + a0 + 2]))
    lon_d = float(np.degrees(ii * dlam))
    return f"level {kk}, lat {lat_d:.2f}, lon {lon_d:.2f}"


def _flow_arrays(flow: CartesianWind, want, dtype, what):
    out = []
    for field in flow.arrays():
        if tuple(int(s) for s in field.shape) != tuple(want):
            raise ValueError(f"the {what} is {tuple(field.shape)} where {tuple(want)} was "
                             "expected")
        if field.dtype != dtype:
            raise ValueError(f"the {what} is {field.dtype} where the grid tables were built "
                             f"for {dtype}")
        if not field.is_cuda:
            raise ValueError(f"the {what} must be CUDA tensors")
        out.append(field.contiguous())
    return out


def lipschitz(wind: CartesianWind, tables: SphericalGridTables, dt_s: float, *,
              extrapolated: CartesianWind | None = None, reference_length_m: float | None = None,
              level_chunk: int = LIPSCHITZ_LEVEL_CHUNK, fused_norms: bool = True,
              window: BandWindow | None = None,
              extrapolated_window: BandWindow | None = None) -> LipschitzDiagnostics:
    """The flow deformation the trajectory has to stay inside
    (trajectory.py:1174-1420): one kernel over every arrival point
    (``sht_sl_lipschitz``) and one read of the reduced numbers.

    ``extrapolated`` is the wind the search reads at the arrival point (None:
    the wind itself).  With a ``window`` the wind holds the band and its halo
    and the diagnostic is taken on the band's rows; a band's ``extrapolated``
    wind holds the rows of ``extrapolated_window`` (the band's rows and one
    row either side).  ``level_chunk`` and ``fused_norms`` are accepted for
    the reference's signature: the kernel takes all levels in one pass."""
    nlev, nrows, nlon = wind.shape
    nlat = tables.nlat
    held = nlat if window is None else window.source_rows
    if (nrows, nlon) != (held, tables.nlon):
        raise ValueError(f"the wind is {(nrows, nlon)} where {(held, tables.nlon)} rows were "
                         f"expected on a {tables.shape} grid")
    rows = slice(0, nlat) if window is None else window.arrival
    ex_held0, ex_rows = (0, nlat) if window is None else (window.source.start, held)
    if extrapolated is not None:
        if window is None:
            if tuple(extrapolated.shape) != tuple(wind.shape):
                raise ValueError(f"the extrapolated wind is {extrapolated.shape} where the wind "
                                 f"is {wind.shape}")
        else:
            if extrapolated_window is None or extrapolated_window.arrival != window.arrival:
                raise ValueError("a band's extrapolated wind needs the window of the rows it "
                                 "holds, computing the band's own rows")
            want = extrapolated_window.source_shape(nlev)
            if tuple(extrapolated.shape) != tuple(want):
                raise ValueError(f"the band's extrapolated wind is {extrapolated.shape} where "
                                 f"{want} was expected")
            ex_held0, ex_rows = extrapolated_window.source.start, extrapolated_window.source_rows
    lref = (tables.equatorial_spacing_m() if reference_length_m is None
            else float(reference_length_m))
    if not np.isfinite(lref) or lref <= 0.0:
        raise ValueError("reference_length_m must be finite and positive")
    if nlev < 2:
        raise ValueError(f"nlev >= 2 is required, got {nlev}")
    # the rows a derivative reads: the band's and one either side (the pole
    # row itself beyond a pole)
    need0 = 0 if rows.start == 0 else rows.start - 1
    need1 = nlat if rows.stop == nlat else rows.stop + 1
    if window is not None:
        for h0, n in ((window.source.start, held),) + (
                ((ex_held0, ex_rows),) if extrapolated is not None else ()):
            if h0 > need0 or h0 + n < need1:
                raise HaloEscape(window, "Lipschitz diagnostic")
    ins = _flow_arrays(wind, wind.shape, tables.dtype, "wind")
    exs = ([None] * 4 if extrapolated is None else
           _flow_arrays(extrapolated, extrapolated.shape, tables.dtype, "extrapolated wind"))
    maxima = (ctypes.c_double * 5)()
    minima = (ctypes.c_double * 2)()
    argmin = (ctypes.c_int64 * 2)()
    src0 = 0 if window is None else window.source.start
    _lib.call("sht_sl_lipschitz", tables._handle, int(nlev), int(rows.start), int(rows.stop),
              *[_ptr(t) for t in ins], int(src0), int(held),
              *[None if t is None else _ptr(t) for t in exs], int(ex_held0), int(ex_rows),
              float(dt_s), float(tables.radius_m), float(lref), maxima, minima, argmin,
              _stream())
    sm, fm, hm, vm, bm = (max(0.0, float(v)) for v in maxima)
    lat_ext = tables.host_tables(4)["lat_ext"]
    shape = (nlev, rows.stop - rows.start, nlon)
    folds = {}
    for side, value, flat in (("departure", minima[0], argmin[0]),
                              ("arrival", minima[1], argmin[1])):
        value = float(value)
        text = _where(int(flat), shape, lat_ext, tables.dlam, rows.start) if value < 2.0 else ""
        folds[side] = (min(1.0, value), text)
    dt = float(dt_s)
    return LipschitzDiagnostics(
        dt_s=dt, reference_length_m=lref, lipschitz=dt * max(hm, vm, bm),
        lipschitz_frobenius=dt * fm, lipschitz_horizontal=dt * hm,
        jacobian_spectral_s=sm, jacobian_frobenius_s=fm, jacobian_horizontal_s=hm,
        lipschitz_vertical=dt * vm, jacobian_vertical_s=vm, lipschitz_mixed=dt * sm,
        lipschitz_balanced=dt * bm, jacobian_balanced_s=bm,
        fold_determinant_arrival=folds["arrival"][0],
        fold_determinant_departure=folds["departure"][0],
        fold_where_arrival=folds["arrival"][1], fold_where_departure=folds["departure"][1])


def convergence(diagnostics: TrajectoryDiagnostics, limit_cells: float) -> None:
    """Refuse a trajectory whose last iteration still moved more than
    ``limit_cells`` of the local meridional grid length
    (trajectory.py:1423-1441)."""
    if diagnostics.move_max_cells > float(limit_cells):
        raise ValueError(
            "the departure-point search did not converge: the last of "
            f"{diagnostics.iterations} iterations still moved a point by "
            f"{diagnostics.move_max_m:.3f} m, which is "
            f"{diagnostics.move_max_cells:.4f} of the local meridional grid "
            f"length against a limit of {float(limit_cells):.4f}; an "
            "unconverged trajectory mislocates the flow and shows no other symptom")


def converged_departure_points(wind: CartesianWind, tables: SphericalGridTables, dt_s: float,
                               *, iterations: int, limit_cells: float,
                               extrapolated: CartesianWind | None = None,
                               window: BandWindow | None = None, defer_escape: bool = False,
                               solver: str = "fixed_point"):
    """The departure points, converged or refused (trajectory.py:1454-1490):
    a search whose last iteration still moved more than ``limit_cells`` is
    run again from the start at ``MAXIMUM_TRAJECTORY_ITERATIONS`` before
    ``convergence`` refuses it; a search that converges at the configured
    count returns its own bits."""
    stencil, diagnostics = departure_points(
        wind, tables, dt_s, iterations=int(iterations), extrapolated=extrapolated,
        window=window, defer_escape=defer_escape, solver=solver)
    if (diagnostics.move_max_cells > float(limit_cells)
            and int(iterations) < MAXIMUM_TRAJECTORY_ITERATIONS):
        del stencil
        stencil, diagnostics = departure_points(
            wind, tables, dt_s, iterations=MAXIMUM_TRAJECTORY_ITERATIONS,
            extrapolated=extrapolated, window=window, defer_escape=defer_escape, solver=solver)
    convergence(diagnostics, limit_cells)
    return stencil, diagnostics


def refuse_trajectory_fold(diagnostics: LipschitzDiagnostics, minimum: float) -> None:
    """Refuse a time step whose trajectory map folds: the fold determinant
    below ``minimum`` (trajectory.py:1511-1560; the same message)."""
    floor = float(minimum)
    if not (0.0 <= floor < 1.0):
        raise ValueError(
            "the minimum fold determinant must lie in [0, 1): zero is the fold itself, and one "
            "would refuse every flow with any divergence or strain at all")
    value = diagnostics.fold_determinant
    if not np.isfinite(value) or value < floor:
        where = (diagnostics.fold_where_departure if diagnostics.fold_side == "departure"
                 else diagnostics.fold_where_arrival)
        raise ValueError(
            f"the trajectory map folds: min det(I - (dt/2) J) over the grid "
            f"reads {diagnostics.fold_determinant_arrival:.4f} on the "
            f"arrival side and det(I + (dt/2) J) "
            f"{diagnostics.fold_determinant_departure:.4f} on the departure "
            f"side at dt = {diagnostics.dt_s:g} s, against a floor of "
            f"{floor:.4f} (binding: {diagnostics.fold_side}, at {where}); at zero two "
            "arrival points share a departure point and the interpolation "
            "samples a folded field, which mislocates the flow silently.  "
            f"The deformation norms, reported and not gated, read "
            f"{diagnostics.lipschitz:.4f} (horizontal "
            f"{diagnostics.lipschitz_horizontal:.4f}, vertical "
            f"{diagnostics.lipschitz_vertical:.4f}, balanced "
            f"{diagnostics.lipschitz_balanced:.4f}).  A shorter [time] dt_s "
            "moves the determinant toward one")
