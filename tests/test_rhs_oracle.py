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


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_elementwise_chains_match_reference(golden, tag):
    """Momentum/Bernoulli, the tracer-flux pair and the scalar tendency against
    the reference's own numpy specifications (tools/gpu_selftest_rhs.py),
    bit for bit: the oracle keeps their association."""
    g = golden("rhs_elementwise.npz")
    f = {k[: -len(tag) - 1]: g[k] for k in g if k.endswith(tag)}
    rgas = f["zeta"].dtype.type(287.0528)
    mu, mv, bern = O.momentum_bernoulli(f["zeta"], f["cor"], f["u"], f["v"], f["wu"], f["wv"],
                                        f["tv"], f["pg"], f["ge"], f["gn"], f["phi"], rgas)
    np.testing.assert_array_equal(mu, f["mu"])
    np.testing.assert_array_equal(mv, f["mv"])
    np.testing.assert_array_equal(bern, f["bern"])
    fx, fy = O.tracer_flux(f["dp"], f["s"], f["u"], f["v"])
    np.testing.assert_array_equal(fx, f["fx"])
    np.testing.assert_array_equal(fy, f["fy"])
    np.testing.assert_array_equal(O.scalar_tendency(f["h"], f["vert"], f["s"], f["dpt"], f["dp"]),
                                  f["st"])
