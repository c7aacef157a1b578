"""Host-side argument logic of the semi-Lagrangian, sampling and RHS
modules: the reference's error texts and shape rules, checked without a GPU
(no library call is made)."""
from __future__ import annotations

import numpy as np
import pytest


def test_sampling_points_and_regular_grid():
    from b200sht.sampling import _points, _resolve_precision, regular_latlon_coordinates

    lat, lon, shape = _points([[0.0, 45.0]], [10.0, 20.0])
    assert shape == (1, 2) and np.allclose(lat, np.deg2rad([0.0, 45.0]))
    with pytest.raises(ValueError, match="finite"):
        _points([np.inf], [0.0])
    with pytest.raises(ValueError, match="latitude must lie"):
        _points([-90.5], [0.0])
    assert _resolve_precision(None) == "float64"
    with pytest.raises(ValueError, match="precision must be one of"):
        _resolve_precision("bfloat16")
    la, lo = regular_latlon_coordinates(4, 8)
    assert np.allclose(la, [-67.5, -22.5, 22.5, 67.5]) and np.allclose(lo, np.arange(8) * 45.0)
    la, _ = regular_latlon_coordinates(3, 4, include_poles=True)
    assert np.allclose(la, [-90.0, 0.0, 90.0])
    with pytest.raises(ValueError, match="nlat>=2 and nlon>=4"):
        regular_latlon_coordinates(1, 8)
    with pytest.raises(ValueError, match="must be integers"):
        regular_latlon_coordinates(True, 8)


def test_semilag_option_rules():
    from b200sht.semilag import _limiter_of, _validate

    assert _limiter_of(True) == "quasi_monotone" and _limiter_of(False) == "none"
    assert _limiter_of("none") == "none"
    _validate("quasi_monotone", True, 4)
    with pytest.raises(ValueError, match="limiter must be one of"):
        _validate("positive_definite", False, 4)
    with pytest.raises(ValueError, match="horizontal order must be one of"):
        _validate("none", False, 8)
    with pytest.raises(ValueError, match="unlimited gather has none"):
        _validate("none", True, 4)
    with pytest.raises(ValueError, match="cubic gather only"):
        _validate("quasi_monotone", True, 6)


def test_band_window_geometry_and_escape_text():
    import types

    from b200sht.semilag import BandWindow, HaloEscape

    tables = types.SimpleNamespace(nlon=64)
    win = BandWindow(tables, slice(8, 24), slice(12, 20), None)
    assert (win.source_rows, win.arrival_rows, win.lead) == (16, 8, 4)
    assert win.local == slice(4, 12)
    assert win.arrival_shape(5) == (5, 8, 64) and win.source_shape(5) == (5, 16, 64)
    err = HaloEscape(win, "gather")
    assert isinstance(err, ValueError)
    assert "rows 12..20" in str(err) and "rows 8..24" in str(err)
