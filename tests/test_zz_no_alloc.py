"""The allocation-free forward transform, sht_forward_static_scratch.

It serves callers that may not allocate device memory when they transform
(host callbacks, allocator hooks, processes whose device memory belongs to
an external manager): the plan is built up front and every call reuses a
fixed buffer compiled into the library.  These checks call it through the C
ABI twice in a row and compare each result with the regular sht_forward on
the same plan, at the tolerances the other parity tests use; they also check
the clear rejection of a call that needs more than the fixed buffer.  The
file sorts last so that a run stopping at the first failure has already run
every other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_l2(a, b):
    w = np.where(np.arange(a.shape[-1]) == 0, 1.0, 2.0)[None, :]
    return float(np.sqrt(np.sum(w * np.abs(a - b) ** 2) / np.sum(w * np.abs(b) ** 2)))


@pytest.mark.parametrize("precision,tol,t,kw", [
    ("float32", 2e-6, 62, dict(nlat=94, nlon=192, dealias_factor=1.49)),
    ("float64", 1e-12, 62, dict(nlat=94, nlon=192, dealias_factor=1.49)),
    ("float32", 2e-6, 255, {}),
])
def test_static_scratch_forward_matches_sht_forward(precision, tol, t, kw):
    import torch

    from b200sht import SphericalHarmonicTransform, build
    from b200sht import _lib
    from b200sht.synthetic import red_spectrum

    build.build()
    lib = _lib.load()
    sht = SphericalHarmonicTransform.create(t, precision=precision, **kw)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    planes = 3
    for call in range(2):
        coeff = red_spectrum(t, planes, seed=100 + call)
        grid = sht.inverse(coeff).contiguous()
        expected = sht.backend.to_numpy(sht.forward(grid))
        out = torch.empty((planes, t + 1, t + 1), dtype=sht.backend.complex_dtype,
                          device=sht.backend.device)
        st = lib.sht_forward_static_scratch(sht.plan.handle, ctypes.c_void_p(grid.data_ptr()),
                                            planes, ctypes.c_void_p(out.data_ptr()), stream)
        _lib.check(st)
        got = sht.backend.to_numpy(out)
        assert _rel_l2(got, expected) <= tol, (precision, call)
        assert np.all(got[..., 0].imag == 0)


def test_static_scratch_rejects_oversize_and_split16():
    import torch

    from b200sht import SphericalHarmonicTransform
    from b200sht import _lib

    lib = _lib.load()
    sht = SphericalHarmonicTransform.create(511, precision="float32")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    grid = torch.zeros((64, 768, 1536), dtype=torch.float32, device=sht.backend.device)
    out = torch.empty((64, 512, 512), dtype=torch.complex64, device=sht.backend.device)
    st = lib.sht_forward_static_scratch(sht.plan.handle, ctypes.c_void_p(grid.data_ptr()), 64,
                                        ctypes.c_void_p(out.data_ptr()), stream)
    assert st == _lib.SHT_ERR_ARG
    msg = lib.sht_last_error().decode()
    assert "above the fixed" in msg and "planes per call" in msg
    split = SphericalHarmonicTransform.create(21, precision="split16")
    g = torch.zeros((1, split.grid.nlat, split.grid.nlon), dtype=torch.float32,
                    device=split.backend.device)
    c = torch.empty((1, 22, 22), dtype=torch.complex64, device=split.backend.device)
    st = lib.sht_forward_static_scratch(split.plan.handle, ctypes.c_void_p(g.data_ptr()), 1,
                                        ctypes.c_void_p(c.data_ptr()), stream)
    assert st == _lib.SHT_ERR_ARG
