"""The plan's Legendre tables read back in the reference's dense layout.

``t._basis.dense()``, ``t._derivative_basis.dense()`` and
``t._analysis.dense()`` are what the reference's bit-identity test compares
with its dense tables (tests/test_global_spectral_bit_identity.py:118-129).
Here they are compared with the oracle's dense tables, which the golden
vectors pin: FP64 within 1e-12 of the table's largest entry (Newton nodes
against leggauss, the within-parity Gram correction against the full solve);
FP32 and split16 hold the FP64 table rounded once to FP32, so within half an
FP32 ulp of each entry plus that.  The vector analysis's weighted tables are
checked through the plan within 1e-11: their weight w / cos(phi) on the rows
next to the poles turns the last-bit differences between the Newton and
leggauss nodes into 2e-12 of the table's largest entry at T62.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (truncation, nlat, nlon): the default grids of T21 (odd nlat: the equator
# row is its own mirror) and T62, and a wider even grid.
GRIDS = [(21, None, None), (62, None, None), (31, 64, 128)]


def _close(have, want, precision, rel=1e-12):
    scale = float(np.max(np.abs(want)))
    tol = rel * scale
    if precision != "float64":
        tol = tol + 2.0 ** -24 * np.abs(want)
    return bool(np.all(np.abs(have.astype(np.float64) - want) <= tol))


def _pair(T, nlat, nlon, precision):
    from b200sht import SphericalHarmonicTransform
    from oracle.dense_sht import DenseSHT

    t = SphericalHarmonicTransform.create(T, nlat=nlat, nlon=nlon, precision=precision)
    return t, DenseSHT(T, t.grid.nlat, t.grid.nlon)


@pytest.mark.parametrize("precision", ["float64", "float32", "split16"])
@pytest.mark.parametrize("T,nlat,nlon", GRIDS)
def test_dense_tables_match_the_oracle(T, nlat, nlon, precision):
    t, ora = _pair(T, nlat, nlon, precision)
    t1, nl = T + 1, t.grid.nlat
    dtype = np.float64 if precision == "float64" else np.float32
    for table, want in ((t._basis, ora.basis_mnj), (t._derivative_basis, ora.dbasis_mnj),
                        (t._analysis, ora.analysis_mjn)):
        have = table.dense()
        assert have.dtype == dtype and have.shape == want.shape, table.name
        assert have.shape == ((t1, nl, t1) if table.layout == "jn" else (t1, t1, nl))
        assert _close(have, want, precision), table.name
        # above the triangle (n < m) every entry is exactly zero
        mi, ni = np.nonzero(np.arange(t1)[:, None] > np.arange(t1)[None, :])
        above = have[mi, ni, :] if table.layout == "nj" else have[mi, :, ni]
        assert not np.any(above), table.name


@pytest.mark.parametrize("T,nlat,nlon", GRIDS)
def test_vector_analysis_tables_match_the_oracle(T, nlat, nlon):
    from b200sht import _lib

    t, ora = _pair(T, nlat, nlon, "float64")
    t1, nl = T + 1, t.grid.nlat
    scale = 2.0 * math.pi / t.grid.radius_m
    rot = t.plan.read_table(_lib.SHT_TABLE_ROTATION, (t1, nl, t1), np.float64)
    shear = t.plan.read_table(_lib.SHT_TABLE_SHEAR, (t1, nl, t1), np.float64)
    w_cos = (ora.w / ora.coslat * scale)[None, :, None]
    assert _close(rot, ora.basis_mnj.transpose(0, 2, 1) * w_cos, "float64", rel=1e-11)
    assert _close(shear, ora.dbasis_mnj.transpose(0, 2, 1) * (ora.w * scale)[None, :, None],
                  "float64", rel=1e-11)


def _folded_elements(T, nlat):
    H = (nlat + 1) // 2
    hx = -(-H // 4) * 4
    syn = ana = 0
    for m in range(T + 1):
        for q in range(2):
            e = max(0, (T - m - q) // 2 + 1)
            syn += e * hx
            ana += H * (-(-e // 4) * 4)
    return syn, ana


def test_table_objects_and_resident_bytes():
    from b200sht import SphericalHarmonicTransform

    t64 = SphericalHarmonicTransform.create(21, precision="float64")
    t32 = SphericalHarmonicTransform.create(21, precision="float32")
    t16 = SphericalHarmonicTransform.create(21, precision="split16")
    # one object per table, equal to its seam name, told apart by identity
    assert t64._basis is t64._basis and t64._analysis is t64._analysis
    assert str(t64._basis) == "basis" and t64._analysis == "analysis"
    assert t64._derivative_basis == "derivative_basis"
    assert len({id(t64._basis), id(t64._analysis), id(t64._derivative_basis)}) == 3
    assert t64._dbasis is t64._derivative_basis
    syn, ana = _folded_elements(21, t64.grid.nlat)
    assert t64.legendre_table_nbytes == {"basis": 8 * syn, "analysis": 8 * ana,
                                         "derivative": 8 * syn, "rotation": 8 * ana,
                                         "shear": 8 * ana, "scratch": 0}
    assert t32.legendre_table_nbytes["basis"] == 4 * syn
    assert t32._analysis.nbytes == 4 * ana
    # split16 holds its FP16 hi/lo tile image beside the FP32 table
    b16 = t16.legendre_table_nbytes
    assert all(b16[k] > t32.legendre_table_nbytes[k] for k in ("basis", "analysis", "derivative"))
    # a table outlives nothing: once the transform is gone it says so
    table = t32._basis
    del t32
    import gc

    gc.collect()
    with pytest.raises(RuntimeError, match="is gone"):
        table.dense()
