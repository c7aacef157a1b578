"""The semi-Lagrangian gather oracle against the reference's own outputs
(tests/golden/sl_gather_*.npz, recorded by make_golden_sl.py from the
reference's numpy gather_batch / gather_linear_batch): the pole-extended
tables of both stencil widths and every (order, limiter, deficit) case."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import sl_gather as O

CASES = [("cubic_qm", 4, "quasi_monotone", False), ("cubic_qm_deficit", 4, "quasi_monotone", True),
         ("cubic_none", 4, "none", False), ("quintic_qm", 6, "quasi_monotone", False),
         ("quintic_none", 6, "none", False)]


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("order", [4, 6])
def test_tables_match_reference(golden, tag, order):
    g = golden(f"sl_gather_{tag}.npz")
    t = O.build_tables(g["lat"], int(g["nlon"]), order)
    for key in ("lat_ext", "mrden", "rowoff", "rowshift", "mlut"):
        ref = g[f"{key}{order}"]
        np.testing.assert_array_equal(t[key], ref.reshape(t[key].shape))


@pytest.mark.parametrize("tag,dtype", [("f64", np.float64), ("f32", np.float32)])
@pytest.mark.parametrize("name,order,limiter,deficit", CASES)
def test_gather_matches_reference(golden, tag, dtype, name, order, limiter, deficit):
    g = golden(f"sl_gather_{tag}.npz")
    out = O.gather(list(g["fields"]), g["xi"], g["phi"], g["level"], g["lat"], int(g["nlon"]),
                   order=order, limiter=limiter, deficit=deficit, dtype=dtype)
    if deficit:
        np.testing.assert_array_equal(np.stack([v for v, _ in out]), g[name])
        np.testing.assert_array_equal(np.stack([c for _, c in out]), g[name + "_cut"])
    else:
        np.testing.assert_array_equal(np.stack(out), g[name])


@pytest.mark.parametrize("tag,dtype", [("f64", np.float64), ("f32", np.float32)])
def test_linear_matches_reference(golden, tag, dtype):
    g = golden(f"sl_gather_{tag}.npz")
    out = O.gather_linear(list(g["fields"]), g["xi"], g["phi"], g["level"], g["lat"],
                          int(g["nlon"]), dtype=dtype)
    np.testing.assert_array_equal(np.stack(out), g["linear"])


def test_deficit_marks_the_clipped_points(golden):
    """The seeded departure points clip some values and leave others: the
    deficit of the limited cubic gather is nonzero at some points, zero at
    the rest, and value + deficit is the unclipped sum."""
    g = golden("sl_gather_f64.npz")
    (v, c), = O.gather([g["fields"][0]], g["xi"], g["phi"], g["level"], g["lat"],
                       int(g["nlon"]), deficit=True)
    assert np.isfinite(v).all() and np.isfinite(c).all()
    assert 0 < np.count_nonzero(c) < c.size
    np.testing.assert_array_equal(v[c == 0], g["cubic_qm"][0][c == 0])


@pytest.mark.parametrize("tag,dtype", [("f64", np.float64), ("f32", np.float32)])
def test_departure_search_matches_reference(golden, tag, dtype):
    g = golden(f"sl_gather_{tag}.npz")
    xi, phi, lev, _, _ = O.departure(list(g["wind"]), g["lat"], int(g["nlon"]), float(g["dt"]),
                                     iterations=3, extrapolated=list(g["wind_ex"]), dtype=dtype)
    np.testing.assert_array_equal(xi, g["dep_xi"])
    np.testing.assert_array_equal(phi, g["dep_phi"])
    np.testing.assert_array_equal(lev, g["dep_level"])
