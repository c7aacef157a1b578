"""Vector spherical-harmonic analysis/synthesis through vorticity/divergence.

Drop-in for the reference's ``VorticityDivergenceOperator``
(src/arwen_global/spectral/vector.py:12-169).  ``wind_from_vordiv`` is one
library call: inverse Laplacian in the pack prologue, one P-synthesis and one
dP/dphi-synthesis of the stacked (psi, chi) pair, and the u/v combination
with its metric factors in the inverse-FFT prologue.  ``vordiv_from_wind`` is
the integration-by-parts analysis (vector.py:54-73, 113-134): one FFT of the
stacked (u, v) pair, the rotational and shear contractions, and the i*m
combination and projection in the unpack epilogue.  Its two halves are also
reachable separately, as in the reference: ``_wind_fourier`` (the waist of
the stacked pair) and ``_vordiv_from_fourier`` / ``vordiv_from_wind_waist`` /
``divergence_from_fourier`` (the contractions of a waist, whole or filled by
bands).  Every contraction passes the transform's ``_batched_contract`` seam
once, with the reference's operand shape, so the reference's census counts
the same calls and planes.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import _lib
from .transform import SphericalHarmonicTransform, _ptr, _stream, fused_operands
from .waist import FourierWaist


@dataclass
class VorticityDivergenceOperator:
    transform: SphericalHarmonicTransform

    def wind_from_vordiv(self, vorticity, divergence):
        """(u, v) from relative vorticity and divergence (vector.py:36-52):
        the reference's gradient of the stacked (psi, chi) pair, two
        contractions of ``(2, *lead)`` planes, fused into one call."""
        t = self.transform
        z = t._spec_in(vorticity)
        d = t._spec_in(divergence)
        if tuple(z.shape) != tuple(d.shape):
            raise ValueError(f"vorticity/divergence shape mismatch: {tuple(z.shape)} != {tuple(d.shape)}")
        lead = tuple(z.shape[:-2])

        def run():
            u = t._empty_grid(lead)
            v = t._empty_grid(lead)
            _lib.call("sht_wind_from_vordiv", t.plan.handle, _ptr(z), _ptr(d), t._planes(z),
                      _ptr(u), _ptr(v), _stream())
            return u, v

        shape = (2, *z.shape)
        op_u, op_v = fused_operands([shape, shape], run)
        with t._contraction_scope():
            u = t._batched_contract(op_u, t._basis)
            v = t._batched_contract(op_v, t._derivative_basis)
        return u, v

    def vordiv_from_wind(self, u, v):
        """Vorticity and divergence of a grid wind by integration by parts
        (vector.py:54-73)."""
        t = self.transform
        uu = t._grid_in(u)
        vv = t._grid_in(v)
        if tuple(uu.shape) != tuple(vv.shape):
            raise ValueError(f"u/v shape mismatch: {tuple(uu.shape)} != {tuple(vv.shape)}")
        lead = tuple(uu.shape[:-2])

        def run():
            zeta = t._empty_spec(lead)
            div = t._empty_spec(lead)
            _lib.call("sht_vordiv_from_wind", t.plan.handle, _ptr(uu), _ptr(vv), t._planes(uu),
                      _ptr(zeta), _ptr(div), _stream())
            return zeta, div

        return self._contract_pair((2, *lead, t.grid.nlat, t.truncation + 1), run)

    def vordiv_from_wind_waist(self, waist: FourierWaist):
        """``vordiv_from_wind`` from a waist a band pipeline filled
        (vector.py:75-82); the waist is read whole."""
        return self._vordiv_from_fourier(waist)

    def _wind_fourier(self, pair, *, bands: int | None = None) -> FourierWaist:
        """The Fourier waist of a stacked ``(2, ..., nlat, nlon)`` wind pair
        (vector.py:84-111): the first half of ``vordiv_from_wind``."""
        return self.transform.fourier_waist(pair, bands=bands)

    def _pair_values(self, fourier, what: str):
        """The ``(2, *lead, nlat, T+1)`` waist values of ``fourier`` (a
        ``FourierWaist``, closed here if a band fill left it open, or a raw
        zonal spectrum at least T+1 orders wide, cut here), contiguous."""
        t = self.transform
        if isinstance(fourier, FourierWaist):
            raw = fourier.close().values
        else:
            raw = t.backend.asarray(fourier, dtype=t.backend.complex_dtype)
        if raw.dim() < 3 or raw.shape[-2] != t.grid.nlat or raw.shape[-1] < t.truncation + 1:
            raise ValueError(f"{what}: the waist must be (2, ..., {t.grid.nlat}, >= "
                             f"{t.truncation + 1}), got {tuple(raw.shape)}")
        if raw.shape[0] != 2:
            raise ValueError(f"{what} reads a stacked (u, v) waist with the pair on the leading "
                             f"axis, got leading length {raw.shape[0]}")
        return raw[..., : t.truncation + 1].contiguous()

    def _vordiv_from_fourier(self, fourier):
        """The contraction half of ``vordiv_from_wind`` (vector.py:113-134):
        the rotational and shear contractions of the stacked waist, two at
        the seam, one library call."""
        t = self.transform
        fm = self._pair_values(fourier, "_vordiv_from_fourier")
        planes = t._planes(fm[0])
        lead = tuple(fm.shape[1:-2])

        def run():
            zeta = t._empty_spec(lead)
            div = t._empty_spec(lead)
            _lib.call("sht_vordiv_from_waist", t.plan.handle, _ptr(fm), planes, _ptr(zeta),
                      _ptr(div), _stream())
            return zeta, div

        return self._contract_pair(tuple(fm.shape), run)

    def divergence_from_fourier(self, fourier):
        """The divergence half of ``_vordiv_from_fourier`` alone
        (vector.py:136-166): ``D = i m rot[u] - shear[v]``, each of the two
        contractions over one component's rows."""
        t = self.transform
        fm = self._pair_values(fourier, "divergence_from_fourier")
        planes = t._planes(fm[0])
        lead = tuple(fm.shape[1:-2])

        def run():
            div = t._empty_spec(lead)
            _lib.call("sht_divergence_from_waist", t.plan.handle, _ptr(fm), planes, _ptr(div),
                      _stream())
            return (div, div)

        shape = tuple(fm.shape[1:])
        op_r, op_s = fused_operands([shape, shape], run)
        with t._contraction_scope():
            t._batched_contract(op_r, t._basis, transposed=True)
            return t._batched_contract(op_s, t._derivative_basis, transposed=True)

    def _contract_pair(self, shape, run):
        """The rotational and shear contractions of a fused vector analysis
        at the seam; returns (vorticity, divergence)."""
        t = self.transform
        op_r, op_s = fused_operands([shape, shape], run)
        with t._contraction_scope():
            zeta = t._batched_contract(op_r, t._basis, transposed=True)
            div = t._batched_contract(op_s, t._derivative_basis, transposed=True)
        return zeta, div

    def flux_curl_divergence(self, eastward_flux, northward_flux):
        return self.vordiv_from_wind(eastward_flux, northward_flux)
