"""Gaussian latitude/longitude grid whose nodes and weights come from the GPU.

Mirror of the reference's ``GaussianGrid`` (src/arwen_global/spectral/grid.py):
the same shape rule and refusal messages (``shape_for``, grid.py:26-94), the
same exactness condition for a truncation the grid did not derive
(``truncated_to``, grid.py:170-201), rows ascending in sin(latitude) with row
0 southernmost.  The nodes and weights are computed in FP64 on the device by
Newton iteration (``sht_plan_create``) instead of ``numpy.polynomial.legendre.
leggauss``; they agree with it to about one unit in the last place.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from dataclasses import dataclass

import numpy as np

from . import _lib

EARTH_RADIUS_M = 6_371_220.0  # src/arwen_global/spectral/constants.py:4


def shape_for(truncation, *, nlat=None, nlon=None, dealias_factor=1.5):
    """``(nlat, nlon)`` for a truncation: ``nlat >= max(T+1, ceil(f (T+1)))``,
    ``nlon >= max(2T+1, ceil(2 f (T+1)))`` rounded up to even; explicit sizes
    below the rule, or an odd explicit nlon, are refused."""
    if isinstance(truncation, bool) or not isinstance(truncation, (int, np.integer)):
        raise ValueError("truncation must be an integer")
    t = int(truncation)
    if t < 1:
        raise ValueError(f"truncation must be >= 1, got {truncation}")
    if isinstance(dealias_factor, bool) or not math.isfinite(dealias_factor) or dealias_factor < 1.0:
        raise ValueError("dealias_factor must be finite and >= 1")
    required_lat = max(t + 1, int(math.ceil(dealias_factor * (t + 1))))
    required_lon = max(2 * t + 1, int(math.ceil(2.0 * dealias_factor * (t + 1))))
    if nlat is None:
        nl = required_lat
    else:
        if isinstance(nlat, bool) or not isinstance(nlat, (int, np.integer)):
            raise ValueError("nlat must be an integer")
        nl = int(nlat)
        if nl < required_lat:
            raise ValueError(
                f"nlat={nl} is too small for T{t} with dealias_factor={dealias_factor:g}; "
                f"need at least {required_lat}")
    if nlon is None:
        no = required_lon + (required_lon % 2)
    else:
        if isinstance(nlon, bool) or not isinstance(nlon, (int, np.integer)):
            raise ValueError("nlon must be an integer")
        no = int(nlon)
        if no % 2:
            raise ValueError(
                "explicit nlon must be even so positive/negative FFT frequencies have one "
                "unambiguous layout")
        if no < required_lon:
            raise ValueError(
                f"nlon={no} is too small for T{t} with dealias_factor={dealias_factor:g}; "
                f"need at least {required_lon} (rounded up to the next even value)")
    return nl, no


def device_geometry(truncation: int, nlat: int, nlon: int, radius_m: float, plan=None):
    """FP64 ``(mu, weights, coslat)`` from a plan (a geometry-only plan when
    none is given)."""
    lib = _lib.load()
    own = plan is None
    if own:
        handle = ctypes.c_void_p()
        _lib.check(lib.sht_plan_create(int(truncation), int(nlat), int(nlon), float(radius_m),
                                       _lib.SHT_PREC_F64, 1, ctypes.byref(handle)))
        plan = handle
    try:
        mu = np.zeros(nlat)
        w = np.zeros(nlat)
        cl = np.zeros(nlat)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(lib.sht_plan_geometry(plan, mu.ctypes.data_as(dp), w.ctypes.data_as(dp),
                                         cl.ctypes.data_as(dp)))
    finally:
        if own:
            lib.sht_plan_destroy(plan)
    return mu, w, cl


@dataclass(frozen=True)
class GaussianGrid:
    truncation: int
    nlat: int
    nlon: int
    sin_lat: np.ndarray
    lat_rad: np.ndarray
    lon_rad: np.ndarray
    quadrature_weights: np.ndarray
    cos_lat: np.ndarray
    radius_m: float = EARTH_RADIUS_M

    shape_for = staticmethod(shape_for)

    @classmethod
    def from_geometry(cls, truncation, nlat, nlon, mu, w, coslat, radius_m=EARTH_RADIUS_M):
        return cls(
            truncation=int(truncation), nlat=int(nlat), nlon=int(nlon),
            sin_lat=np.asarray(mu, np.float64), lat_rad=np.arcsin(mu),
            lon_rad=np.arange(nlon, dtype=np.float64) * (2.0 * np.pi / nlon),
            quadrature_weights=np.asarray(w, np.float64),
            cos_lat=np.asarray(coslat, np.float64), radius_m=float(radius_m))

    @classmethod
    def create(cls, truncation, *, nlat=None, nlon=None, dealias_factor=1.5,
               radius_m=EARTH_RADIUS_M):
        nl, no = shape_for(truncation, nlat=nlat, nlon=nlon, dealias_factor=dealias_factor)
        if not math.isfinite(radius_m) or radius_m <= 0:
            raise ValueError("radius_m must be finite and positive")
        mu, w, cl = device_geometry(int(truncation), nl, no, radius_m)
        return cls.from_geometry(truncation, nl, no, mu, w, cl, radius_m)

    @classmethod
    def for_shape(cls, nlat, nlon, *, radius_m=EARTH_RADIUS_M):
        return cls.create(int(nlon) // 2 - 1, nlat=nlat, nlon=nlon, dealias_factor=1.0,
                          radius_m=radius_m)

    @property
    def shape(self):
        return self.nlat, self.nlon

    @property
    def zonal_content_truncation(self):
        return self.nlon // 2 - 1

    @property
    def exact_analysis_truncation(self):
        t_in = self.zonal_content_truncation
        return min(t_in, 2 * self.nlat - 1 - t_in)

    def truncated_to(self, truncation):
        """This grid's nodes under a truncation it did not derive; refuses an
        aliased projection (grid.py:170-201)."""
        if isinstance(truncation, bool) or not isinstance(truncation, (int, np.integer)):
            raise ValueError("truncation must be an integer")
        t = int(truncation)
        if t < 1:
            raise ValueError(f"truncation must be >= 1, got {truncation}")
        t_in = self.zonal_content_truncation
        if t > t_in:
            raise ValueError(
                f"T{t} exceeds the zonal content of a {self.nlat}x{self.nlon} grid: the real "
                f"FFT of {self.nlon} longitudes carries orders m <= nlon/2 - 1 = {t_in}, so "
                f"order {t} does not exist there")
        if t_in + t > 2 * self.nlat - 1:
            raise ValueError(
                f"T{t} on a {self.nlat}x{self.nlon} grid is not an exact projection: the "
                f"exactness condition T_in + T <= 2*nlat - 1 with T_in = nlon/2 - 1 = {t_in} "
                f"reads {t_in} + {t} = {t_in + t} > {2 * self.nlat - 1}; "
                f"T <= {self.exact_analysis_truncation} is exact on this grid")
        return dataclasses.replace(self, truncation=t)

    @property
    def latitude_deg(self):
        return np.rad2deg(self.lat_rad)

    @property
    def longitude_deg(self):
        return np.rad2deg(self.lon_rad)

    def mesh(self):
        lon, lat = np.meshgrid(self.lon_rad, self.lat_rad)
        return lat, lon

    def global_mean(self, field) -> float:
        arr = np.asarray(field, dtype=np.float64)
        if arr.shape[-2:] != self.shape:
            raise ValueError(f"field has shape {arr.shape[-2:]}, expected {self.shape}")
        return float(0.5 * np.sum(arr.mean(axis=-1) * self.quadrature_weights, axis=-1))

    def global_integral(self, field) -> float:
        return 4.0 * np.pi * self.global_mean(field)

    def rms(self, field) -> float:
        arr = np.asarray(field, dtype=np.float64)
        return math.sqrt(max(0.0, self.global_mean(arr * arr)))

    def degree_length_m(self, degree: int) -> float:
        """The wavelength of total degree ``degree`` along a great circle,
        2 pi a / n (infinite at n = 0; grid.py:229-231)."""
        n = int(degree)
        return math.inf if n == 0 else 2.0 * math.pi * self.radius_m / n
