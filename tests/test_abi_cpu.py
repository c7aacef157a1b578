"""Host-side checks that need no GPU: the C ABI library loads, exports every
symbol the public header declares, and validates arguments before touching
CUDA; the Python shape rules match the reference's."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden


def _header_symbols():
    text = (ROOT / "include" / "b200sht.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(sht_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    from b200sht import build, _lib

    build.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    from b200sht import _lib

    names = _header_symbols()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name
    assert set(_lib.SIGNATURES) == set(names)
    assert lib.sht_abi_version() == _lib.SHT_ABI_VERSION


def test_plan_create_validates_before_cuda(lib):
    from b200sht import _lib

    h = ctypes.c_void_p()
    cases = [
        (0, 4, 8, 1.0, 0, 0),        # truncation < 1
        (10, 5, 40, 1.0, 0, 0),      # nlat < T+1
        (10, 16, 31, 1.0, 0, 0),     # odd nlon
        (10, 16, 20, 1.0, 0, 0),     # nlon < 2T+2
        (10, 16, 32, -1.0, 0, 0),    # radius
        (10, 16, 32, 1.0, 7, 0),     # precision
        (10, 16, 32, 1.0, 0, 8),     # flags
    ]
    for args in cases:
        st = lib.sht_plan_create(*args, ctypes.byref(h))
        assert st == _lib.SHT_ERR_ARG, args
        assert lib.sht_last_error()
        assert not h.value
    with pytest.raises(ValueError, match="nlat must be"):
        _lib.check(lib.sht_plan_create(10, 5, 40, 1.0, 0, 0, ctypes.byref(h)))


def test_null_plan_is_an_argument_error(lib):
    from b200sht import _lib

    assert lib.sht_forward(None, None, 1, None, None) == _lib.SHT_ERR_ARG
    assert b"NULL" in lib.sht_last_error()
    assert lib.sht_plan_destroy(None) == _lib.SHT_OK


def test_shape_rule_matches_reference():
    from b200sht.grid import shape_for
    from oracle.dense_sht import grid_shape

    for t in (1, 7, 9, 15, 21, 62, 126, 255, 511):
        assert shape_for(t) == grid_shape(t)
    assert shape_for(62, nlat=94, nlon=192, dealias_factor=1.49) == (94, 192)
    assert shape_for(255) == (384, 768)
    assert shape_for(511) == (768, 1536)
    assert shape_for(126) == (191, 382)
    assert shape_for(126, nlat=192, nlon=384) == (192, 384)
    with pytest.raises(ValueError, match="nlat=94 is too small"):
        shape_for(62, nlat=94)
    with pytest.raises(ValueError, match="explicit nlon must be even"):
        shape_for(10, nlon=41)
    for name in ("sht_t9.npz", "sht_t21.npz", "sht_t62.npz"):
        g = load_golden(name)
        kw = {"nlat": int(g["nlat"]), "nlon": int(g["nlon"])} if name == "sht_t62.npz" else {}
        assert shape_for(int(g["truncation"]), dealias_factor=float(g["dealias_factor"]), **kw) == (
            int(g["nlat"]), int(g["nlon"]))


def test_vertical_operator_modes_match_reference_fixture():
    from b200sht.semi_implicit import VerticalModeOperator

    g = load_golden("helmholtz_t21_l40.npz")
    op = VerticalModeOperator(g["b_matrix"], g["c_matrix"])
    np.testing.assert_allclose(op.eigenvalues, g["eigenvalues"], rtol=1e-10)
    # Eigenvectors agree up to a per-column sign/scale: compare the projectors.
    v_ref = g["eigenvectors"]
    for j in range(op.nlev):
        a = op.eigenvectors[:, j] / np.linalg.norm(op.eigenvectors[:, j])
        b = v_ref[:, j] / np.linalg.norm(v_ref[:, j])
        assert abs(abs(a @ b) - 1.0) < 1e-8


def test_latitude_band_edges_tile_the_grid():
    from b200sht import latitude_band_edges

    assert latitude_band_edges(7, 3) == [(0, 2), (2, 4), (4, 7)]
    assert latitude_band_edges(3, 5) == [(0, 1), (1, 2), (2, 3)]  # empty bands dropped
    for nlat in (1, 32, 94, 768):
        for bands in (1, 2, 7, 100):
            edges = latitude_band_edges(nlat, bands)
            assert edges[0][0] == 0 and edges[-1][1] == nlat
            assert all(a < b for a, b in edges)
            assert all(edges[i][1] == edges[i + 1][0] for i in range(len(edges) - 1))
    with pytest.raises(ValueError):
        latitude_band_edges(0, 1)
    with pytest.raises(ValueError):
        latitude_band_edges(10, 0)
