"""b200sht: the spherical-harmonic transform pair of the ArWen Global sl_si
dycore on a B200 (sm_100a), behind the reference's Python API.

``SphericalHarmonicTransform``, ``VorticityDivergenceOperator`` and
``VerticalModeSemiImplicit`` mirror ``arwen_global.spectral.transform``,
``arwen_global.spectral.vector`` and ``arwen_global.semi_implicit``; every
transform runs in the CUDA library ``lib/libb200sht.so`` through its C ABI.
"""
from .grid import GaussianGrid, shape_for
from .transform import SphericalHarmonicTransform
from .vector import VorticityDivergenceOperator
from .semi_implicit import SpectralState, VerticalModeOperator, VerticalModeSemiImplicit
from .batch import TransformBatch
from .waist import FourierWaist, latitude_band_edges
from .step import DycoreTransformStep

__all__ = [
    "GaussianGrid",
    "shape_for",
    "SphericalHarmonicTransform",
    "VorticityDivergenceOperator",
    "SpectralState",
    "VerticalModeOperator",
    "VerticalModeSemiImplicit",
    "TransformBatch",
    "FourierWaist",
    "latitude_band_edges",
    "DycoreTransformStep",
]
