"""Transforms on the native verification grids with every table resident:
T767 on 1152 x 2304 and T1534 on the 1536 x 3072 linear grid (the reference
streams its tables there), split16 against the FP64 plan and through a
round trip (2e-6, the split bar), FP64 round trip within 1e-12."""
from __future__ import annotations

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_t767_native_grid_round_trip_and_fp64_agreement():
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import CONTROL_SEED, red_spectrum

    T, nl, no = 767, 1152, 2304
    split = SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, precision="split16")
    f64 = SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, precision="float64")
    c64 = torch.as_tensor(red_spectrum(T, 3, CONTROL_SEED), device="cuda")
    g64 = f64.inverse(c64)
    assert float((f64.forward(g64) - c64).abs().max() / c64.abs().max()) < 1e-12
    c = c64.to(split.backend.complex_dtype)
    g = split.inverse(c)
    assert float((g.double() - g64).abs().max() / g64.abs().max()) < 2e-6
    c2 = split.forward(g64.float()).to(torch.complex128)
    assert float((c2 - c64).abs().max() / c64.abs().max()) < 2e-6


def test_t1534_linear_grid_round_trip_and_fp64_agreement():
    """T1534 on 1536 x 3072 (dealias factor 1): the two plans together hold
    about 70 GB of resident tables; two planes."""
    import gc

    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import CONTROL_SEED, red_spectrum

    T, nl, no = 1534, 1536, 3072
    f64 = SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, dealias_factor=1.0,
                                            precision="float64")
    c64 = torch.as_tensor(red_spectrum(T, 2, CONTROL_SEED), device="cuda")
    g64 = f64.inverse(c64)
    assert float((f64.forward(g64) - c64).abs().max() / c64.abs().max()) < 1e-12
    f64.check_device()
    del f64
    gc.collect()
    torch.cuda.empty_cache()
    split = SphericalHarmonicTransform.create(T, nlat=nl, nlon=no, dealias_factor=1.0,
                                              precision="split16")
    g = split.inverse(c64.to(split.backend.complex_dtype))
    assert float((g.double() - g64).abs().max() / g64.abs().max()) < 2e-6
    c2 = split.forward(g64.float()).to(torch.complex128)
    w = torch.ones(T + 1, dtype=torch.float64, device="cuda")
    w[1:] = 2.0
    rel = torch.sqrt(((c2 - c64).abs() ** 2 * w).sum() / (c64.abs() ** 2 * w).sum())
    assert float(rel) < 2e-6
    split.check_device()
    del split
    gc.collect()
    torch.cuda.empty_cache()
