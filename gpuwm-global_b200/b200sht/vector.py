"""Vector spherical-harmonic analysis/synthesis through vorticity/divergence.

Drop-in for the reference's ``VorticityDivergenceOperator``
(src/arwen_global/spectral/vector.py:12-169).  ``wind_from_vordiv`` is one
library call: inverse Laplacian in the pack prologue, one P-synthesis and one
dP/dphi-synthesis of the stacked (psi, chi) pair, and the u/v combination
with its metric factors in the inverse-FFT prologue.  ``vordiv_from_wind`` is
the integration-by-parts analysis (vector.py:54-73, 113-134): one FFT of the
stacked (u, v) pair, the rotational and shear contractions, and the i*m
combination and projection in the unpack epilogue.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import _lib
from .transform import SphericalHarmonicTransform, _ptr, _stream


@dataclass
class VorticityDivergenceOperator:
    transform: SphericalHarmonicTransform

    def wind_from_vordiv(self, vorticity, divergence):
        t = self.transform
        z = t._spec_in(vorticity)
        d = t._spec_in(divergence)
        if tuple(z.shape) != tuple(d.shape):
            raise ValueError(f"vorticity/divergence shape mismatch: {tuple(z.shape)} != {tuple(d.shape)}")
        u = t._empty_grid(z.shape[:-2])
        v = t._empty_grid(z.shape[:-2])
        t.contraction_count += 2
        _lib.call("sht_wind_from_vordiv", t.plan.handle, _ptr(z), _ptr(d), t._planes(z),
                  _ptr(u), _ptr(v), _stream())
        return u, v

    def vordiv_from_wind(self, u, v):
        t = self.transform
        uu = t._grid_in(u)
        vv = t._grid_in(v)
        if tuple(uu.shape) != tuple(vv.shape):
            raise ValueError(f"u/v shape mismatch: {tuple(uu.shape)} != {tuple(vv.shape)}")
        zeta = t._empty_spec(uu.shape[:-2])
        div = t._empty_spec(uu.shape[:-2])
        t.contraction_count += 2
        _lib.call("sht_vordiv_from_wind", t.plan.handle, _ptr(uu), _ptr(vv), t._planes(uu),
                  _ptr(zeta), _ptr(div), _stream())
        return zeta, div

    def flux_curl_divergence(self, eastward_flux, northward_flux):
        return self.vordiv_from_wind(eastward_flux, northward_flux)
