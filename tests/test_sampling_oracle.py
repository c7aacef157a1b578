"""The point-sampling oracle against the reference's recorded host path."""
from __future__ import annotations

import numpy as np

from oracle import sampling as O


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_sampling_matches_reference(golden):
    g = golden("sampling_t21.npz")
    r = float(g["radius"])
    assert _rel(O.sample(g["coeff"], g["lat"], g["lon"]), g["scalar"]) < 1e-13
    e, n = O.sample(g["coeff"], g["lat"][2:], g["lon"][2:], gradient=True, radius=r)
    assert _rel(e, g["east"]) < 1e-13 and _rel(n, g["north"]) < 1e-13
    pe, pn = O.sample(O.inverse_laplacian(g["coeff"][0], r), g["lat"][2:], g["lon"][2:],
                      gradient=True, radius=r)
    ce, cn = O.sample(O.inverse_laplacian(g["coeff"][1], r), g["lat"][2:], g["lon"][2:],
                      gradient=True, radius=r)
    assert _rel(-pn + ce, g["u"]) < 1e-13 and _rel(pe + cn, g["v"]) < 1e-13


def test_triangle_index_is_the_packed_order():
    """Order-major, n fastest inside each order (the reference's
    sampling.py:72-80), with the row of (n, m) at m (T+1) - m (m-1)/2 + n - m."""
    from b200sht.sampling import triangle_index

    for t in (0, 1, 7, 30):
        n, m = triangle_index(t)
        assert n.size == m.size == (t + 1) * (t + 2) // 2
        rows = m * (t + 1) - m * (m - 1) // 2 + (n - m)
        assert np.array_equal(rows, np.arange(n.size)) and np.all(n >= m) and np.all(n <= t)
