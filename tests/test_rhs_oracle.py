"""The RHS oracle's van Leer vertical flux divergence against the
reference's own numpy method (tests/golden/rhs_vertical_flux.npz)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import rhs as O


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_vertical_flux_divergence_matches_reference(golden, tag):
    g = golden("rhs_vertical_flux.npz")
    out = O.vertical_flux_divergence(g[f"s_{tag}"], g[f"w_{tag}"], g[f"pf_{tag}"], g[f"ph_{tag}"])
    np.testing.assert_array_equal(out, g[f"out_{tag}"])


def test_flux_form_conserves_the_column_mass():
    """Interface fluxes telescope: the column sum of the divergence is the
    boundary flux difference, zero here."""
    s, w, pf, ph = O.column_state(10, 3, 4, 2, 7)
    out = O.vertical_flux_divergence(s, w, pf, ph)
    assert np.max(np.abs(out.sum(axis=-3))) < 1e-12 * np.max(np.abs(out))
