"""The allocation-free forward transform, sht_forward_static_scratch.

It serves callers that may not allocate device memory when they transform
(host callbacks, allocator hooks, processes whose device memory belongs to
an external manager): the plan is built up front and every call reuses a
fixed buffer compiled into the library.  These checks call it through the C
ABI on a freshly created plan whose own scratch has never been grown, check
that the device's free memory does not move across those calls (no
allocation), and compare each of two calls in a row with the regular
sht_forward on the same plan.  Both run the same kernels in the same order,
so the results must be equal bit for bit.  They also check the clear
rejection of a call that needs more than the fixed buffer.  The file sorts
last so that a run stopping at the first failure has already run every
other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_forward(lib, sht, grid, planes, t, stream):
    import torch

    out = torch.empty((planes, t + 1, t + 1), dtype=sht.backend.complex_dtype,
                      device=sht.backend.device)
    st = lib.sht_forward_static_scratch(sht.plan.handle, ctypes.c_void_p(grid.data_ptr()),
                                        planes, ctypes.c_void_p(out.data_ptr()), stream)
    return st, out


@pytest.mark.parametrize("precision,t,kw", [
    ("float32", 62, dict(nlat=94, nlon=192, dealias_factor=1.49)),
    ("float64", 62, dict(nlat=94, nlon=192, dealias_factor=1.49)),
    ("float32", 255, {}),
])
def test_static_scratch_forward_matches_sht_forward(precision, t, kw):
    import torch

    from b200sht import SphericalHarmonicTransform, build
    from b200sht import _lib
    from b200sht.synthetic import red_spectrum

    build.build()
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    planes = 3
    grids = []
    # Inputs, and one warm-up call on another plan of the same shape: the
    # kernels' first launches (lazy module loading) and the one-time lookup
    # of the buffer's address happen there, not inside the measured calls.
    warm = SphericalHarmonicTransform.create(t, precision=precision, **kw)
    for call in range(2):
        grids.append(warm.inverse(red_spectrum(t, planes, seed=100 + call)).contiguous())
    _lib.check(_static_forward(lib, warm, grids[0], planes, t, stream)[0])
    sht = SphericalHarmonicTransform.create(t, precision=precision, **kw)
    outs = [torch.empty((planes, t + 1, t + 1), dtype=sht.backend.complex_dtype,
                        device=sht.backend.device) for _ in range(2)]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for call in range(2):
        st = lib.sht_forward_static_scratch(sht.plan.handle,
                                            ctypes.c_void_p(grids[call].data_ptr()), planes,
                                            ctypes.c_void_p(outs[call].data_ptr()), stream)
        _lib.check(st)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before, "the static-scratch calls allocated"
    for call in range(2):
        expected = sht.backend.to_numpy(sht.forward(grids[call]))
        got = sht.backend.to_numpy(outs[call])
        assert np.array_equal(got, expected), (precision, call)
        assert np.all(got[..., 0].imag == 0)


def test_static_scratch_rejects_oversize_and_split16():
    import torch

    from b200sht import SphericalHarmonicTransform
    from b200sht import _lib

    lib = _lib.load()
    sht = SphericalHarmonicTransform.create(511, precision="float32")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    grid = torch.zeros((64, 768, 1536), dtype=torch.float32, device=sht.backend.device)
    st, _ = _static_forward(lib, sht, grid, 64, 511, stream)
    assert st == _lib.SHT_ERR_ARG
    msg = lib.sht_last_error().decode()
    assert "above the fixed" in msg and "planes per call" in msg
    split = SphericalHarmonicTransform.create(21, precision="split16")
    g = torch.zeros((1, split.grid.nlat, split.grid.nlon), dtype=torch.float32,
                    device=split.backend.device)
    st, _ = _static_forward(lib, split, g, 1, 21, stream)
    assert st == _lib.SHT_ERR_ARG
