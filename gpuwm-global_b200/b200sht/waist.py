"""The Fourier waist: the named buffer between the longitude FFT and the
Legendre contraction, in the reference's layout ``(*lead, nlat, T+1)``.

Mirror of ``FourierWaist`` and of the transform's waist methods
(src/arwen_global/spectral/transform.py:68-97, 417-629, 1276-1404,
1435-1473, 1629-1735, 1770-1796): ``open_waist``/``fill_band``/``close``
for band pipelines, ``fourier_waist``, ``contract_waist``,
``contract_values``, ``contract_to_waist``, ``waist_band_to_grid``,
``waist_to_grid``, ``gradient_waists`` and ``gradient_band``, with the
reference's consume-once (``take``) and band-schedule semantics.  Each
conversion is one C-ABI call (``sht_fourier_waist``, ``sht_contract_waist``,
``sht_contract_to_waist``, ``sht_waist_to_grid``).

What differs: the engine's longitude FFT works on latitude pairs (a row and
its mirror), so a band fill is staged on the device and the whole field is
transformed when the waist is closed, and a band drain transforms the whole
waist once (on the first band) and hands out rows of that grid.  The bytes
of every row are therefore those of the whole-field call, whatever the band
schedule -- the reference's bit-identity argument, kept by construction.
On a 180 GB B200 the full grid of any configured workload fits, so the band
schedule is a calling convention here, not a memory saving.
"""
from __future__ import annotations

import torch

from . import _lib
from .transform import SphericalHarmonicTransform, _ptr, _stream, fused_operands

BASIS = "basis"
DERIVATIVE_BASIS = "derivative_basis"
ANALYSIS = "analysis"
_TABLE_CODE = {None: _lib.SHT_WAIST_BASIS, BASIS: _lib.SHT_WAIST_BASIS,
               DERIVATIVE_BASIS: _lib.SHT_WAIST_DBASIS}


def latitude_band_edges(nlat: int, bands: int) -> list[tuple[int, int]]:
    """The band schedule ``floor(k nlat / B)``, ``k = 0..B``, empty bands
    dropped (transform.py:68-97)."""
    n, b = int(nlat), int(bands)
    if n < 1:
        raise ValueError(f"nlat must be >= 1, got {nlat}")
    if b < 1:
        raise ValueError(f"bands must be >= 1, got {bands}")
    cuts = [(k * n) // b for k in range(b + 1)]
    return [(a, c) for a, c in zip(cuts, cuts[1:]) if c > a]


class _RowsFilled:
    """Which latitude rows a band pipeline has written."""

    def __init__(self, nlat: int):
        self.nlat = int(nlat)
        self.rows = torch.zeros(self.nlat, dtype=torch.bool)

    def claim(self, r0: int, r1: int) -> None:
        if not 0 <= r0 < r1 <= self.nlat:
            raise ValueError(f"band [{r0}, {r1}) is not inside [0, {self.nlat})")
        if bool(self.rows[r0:r1].any()):
            raise ValueError(f"band [{r0}, {r1}) overlaps rows already filled")
        self.rows[r0:r1] = True

    def require_complete(self) -> None:
        missing = (~self.rows).nonzero().flatten().tolist()
        if missing:
            raise RuntimeError(f"the waist has {len(missing)} unwritten latitude rows "
                               f"(first {missing[:8]}): a band schedule skipped them")


class FourierWaist:
    """``(*lead, nlat, T+1)`` complex on the device: the zonal spectrum of a
    grid field divided by nlon and cut at ``m = T`` (analysis), or the
    Legendre contraction's output before the inverse FFT (synthesis)."""

    def __init__(self, transform: SphericalHarmonicTransform, values, edges):
        self.transform = transform
        self._values = values
        self._open = False
        self._filled = None
        self._staging = None
        self._grid = None
        self.edges = list(edges)
        self.lead = tuple(values.shape[:-2])
        self.shape = tuple(values.shape)
        self.nbytes = int(values.numel() * values.element_size())

    @classmethod
    def open(cls, transform: SphericalHarmonicTransform, lead, edges) -> "FourierWaist":
        t = transform
        waist = cls.__new__(cls)
        waist.transform = t
        waist.lead = tuple(int(v) for v in lead)
        waist.shape = (*waist.lead, t.grid.nlat, t.truncation + 1)
        waist.edges = list(edges)
        waist._values = None
        waist._open = True
        waist._filled = _RowsFilled(t.grid.nlat)
        waist._staging = t._empty_grid(waist.lead)
        waist._grid = None
        waist.nbytes = int(torch.Size(waist.shape).numel() *
                           torch.empty((), dtype=t.backend.complex_dtype).element_size())
        return waist

    def fill_band(self, r0: int, r1: int, rows) -> None:
        """Write one latitude band of grid space (``(*lead, r1-r0, nlon)``)."""
        if not self._open:
            raise RuntimeError("this FourierWaist was not opened for a band fill: a waist "
                               "built from a whole field is already full")
        t = self.transform
        r0, r1 = int(r0), int(r1)
        f = t.backend.asarray(rows, dtype=t.backend.float_dtype)
        if tuple(f.shape) != (*self.lead, r1 - r0, t.grid.nlon):
            raise ValueError(f"band rows {tuple(f.shape)} are not the waist's "
                             f"{(*self.lead, r1 - r0, t.grid.nlon)}")
        self._filled.claim(r0, r1)
        self._staging[..., r0:r1, :] = f

    def close(self) -> "FourierWaist":
        """Refuse a waist with an unwritten row, then transform it."""
        if self._open:
            t = self.transform
            exchange = getattr(t, "row_exchange", None)
            if (exchange is not None and int(getattr(exchange, "world", 1)) > 1
                    and not bool(self._filled.rows.all())):
                # The rows other cards hold arrive through the card layer
                # (transform.py:547-563); the staged band rows are grid rows.
                exchange.fill_rows(t.backend.xp, self._staging, self._staging.ndim - 2,
                                   name="waist")
                self._filled.rows[:] = True
            self._filled.require_complete()
            out = torch.empty(self.shape, dtype=t.backend.complex_dtype, device=t.backend.device)
            _lib.call("sht_fourier_waist", t.plan.handle, _ptr(self._staging),
                      t._planes(self._staging), _ptr(out), _stream())
            self._values = out
            self._staging = None
            self._open = False
        return self

    @property
    def bands(self) -> int:
        return len(self.edges)

    @property
    def values(self):
        if self._values is None:
            raise RuntimeError("this FourierWaist was consumed: its buffer was handed to a "
                               "drain and released.  Build a new waist instead")
        return self._values

    def take(self):
        """Hand the buffer over and forget it."""
        values = self.values
        self._values = None
        return values

    def band(self, r0: int, r1: int):
        """The waist rows of one latitude band, a view."""
        return self.values[..., int(r0):int(r1), :]

    def drain_scratch(self, rows: int):
        """A zero ``(*lead, rows, nlon//2 + 1)`` half spectrum on the device
        for one band (transform.py:608-630): the orders above T stay the
        zeros an inverse real FFT reads as the spectrum's vanishing tail.
        A fresh buffer per call.  The engine's own drains
        (``waist_band_to_grid``) run the FFT in the library and need none;
        this is for a caller that drains a band itself."""
        t = self.transform
        return torch.zeros((*self.lead, int(rows), t.grid.nlon // 2 + 1),
                           dtype=t.backend.complex_dtype, device=t.backend.device)


# ----------------------------------------------------------------- methods
def open_waist(self, lead, *, bands: int | None = None) -> FourierWaist:
    return FourierWaist.open(self, lead, latitude_band_edges(
        self.grid.nlat, self.latitude_bands if bands is None else bands))


def fourier_waist(self, field, *, bands: int | None = None) -> FourierWaist:
    f = self._grid_in(field)
    out = torch.empty((*f.shape[:-2], self.grid.nlat, self.truncation + 1),
                      dtype=self.backend.complex_dtype, device=self.backend.device)
    _lib.call("sht_fourier_waist", self.plan.handle, _ptr(f), self._planes(f), _ptr(out),
              _stream())
    return FourierWaist(self, out, latitude_band_edges(
        self.grid.nlat, self.latitude_bands if bands is None else bands))


def contract_values(self, values, table=None):
    """The analysis tail on a waist's buffer or a leading slice of it
    (transform.py:1455-1472): one contraction at the seam."""
    if table not in (None, ANALYSIS):
        raise ValueError("the analysis contraction reads the Gram-solved analysis table")
    with self._contraction_scope():
        out = self._batched_contract(values, ANALYSIS, realify=True)
    self._agree_across_cards("analysis", ANALYSIS, out)
    return out


def contract_waist(self, waist: FourierWaist, table=None):
    return self.contract_values(waist.close().take(), table)


def contract_to_waist(self, coeff, table=None, *, bands: int | None = None) -> FourierWaist:
    if table not in _TABLE_CODE:
        raise ValueError(f"table must be one of {sorted(k for k in _TABLE_CODE if k)}")
    return _contract_to_waist(self, coeff, _TABLE_CODE[table], bands)


def _contract_to_waist(self, coeff, code, bands):
    """One synthesis contraction at the seam (transform.py:1629-1652); the
    zonal form (basis times i m, which the reference applies to the
    coefficients first) runs fused."""
    c = self._spec_in(coeff)
    table = DERIVATIVE_BASIS if code == _lib.SHT_WAIST_DBASIS else BASIS
    if code == _lib.SHT_WAIST_ZONAL:
        def run():
            out = torch.empty((*c.shape[:-2], self.grid.nlat, self.truncation + 1),
                              dtype=self.backend.complex_dtype, device=self.backend.device)
            _lib.call("sht_contract_to_waist", self.plan.handle, _ptr(c), self._planes(c),
                      int(code), _ptr(out), _stream())
            return (out,)

        (values,) = fused_operands([tuple(c.shape)], run)
    else:
        values = c
    with self._contraction_scope():
        out = self._batched_contract(values, table)
    self._agree_across_cards("synthesis", table, out)
    return FourierWaist(self, out, latitude_band_edges(
        self.grid.nlat, self.latitude_bands if bands is None else bands))


def _waist_grid(self, values):
    v = values.contiguous()
    out = self._empty_grid(v.shape[:-2])
    _lib.call("sht_waist_to_grid", self.plan.handle, _ptr(v), self._planes(v), _ptr(out),
              _stream())
    return out


def waist_band_to_grid(self, waist: FourierWaist, r0: int, r1: int):
    """One latitude band of a waist in grid space, without consuming it."""
    if waist._grid is None:
        waist._grid = _waist_grid(self, waist.close().values)
    return waist._grid[..., int(r0):int(r1), :]


def waist_to_grid(self, waist: FourierWaist):
    """The whole waist in grid space; consumes the waist."""
    waist.close()
    if waist._grid is not None:
        grid = waist._grid
        waist.take()
        waist._grid = None
        return grid
    return _waist_grid(self, waist.take())


def gradient_waists(self, coeff, *, bands: int | None = None):
    """The two syntheses of ``gradient`` before their drains: the basis times
    i m (eastward) and the d/dphi basis (northward)."""
    return (_contract_to_waist(self, coeff, _lib.SHT_WAIST_ZONAL, bands),
            _contract_to_waist(self, coeff, _lib.SHT_WAIST_DBASIS, bands))


def gradient_band(self, waists, r0: int, r1: int):
    """One latitude band of ``gradient``, drained from ``gradient_waists``."""
    east_waist, north_waist = waists
    r0, r1 = int(r0), int(r1)
    coslat = torch.as_tensor(self.grid.cos_lat[r0:r1], dtype=self.backend.float_dtype,
                             device=self.backend.device)
    east = waist_band_to_grid(self, east_waist, r0, r1) / (self.grid.radius_m * coslat[:, None])
    north = waist_band_to_grid(self, north_waist, r0, r1) / self.grid.radius_m
    return east, north


for _name, _fn in (("open_waist", open_waist), ("fourier_waist", fourier_waist),
                   ("contract_values", contract_values), ("contract_waist", contract_waist),
                   ("contract_to_waist", contract_to_waist),
                   ("waist_band_to_grid", waist_band_to_grid), ("waist_to_grid", waist_to_grid),
                   ("gradient_waists", gradient_waists), ("gradient_band", gradient_band)):
    setattr(SphericalHarmonicTransform, _name, _fn)
