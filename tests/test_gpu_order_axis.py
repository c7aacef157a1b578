"""The order axis and the streamed forms of the transform.

``forward_orders`` / ``inverse_orders`` (the reference's
transform.py:1532-1599) with an order exchange of two ranks: this rank's
columns go through the exchange's ``gather_columns`` and the result is the
single-card result bit for bit.  The other rank is stood in for by a fake
exchange holding the columns that rank would send (the same engine's whole
answer), so the test checks which columns this rank contributes, the names
and shapes it hands the exchange, and that the pieces are placed, not
added.  ``forward_streaming`` / ``inverse_streaming`` return the resident
bits (tests/test_global_spectral_streaming.py:47-80, 179-186 in the
reference).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


class TwoRankOrderExchange:
    """Rank ``rank`` of a two-rank order exchange split at order ``split``;
    ``other`` maps a gather name to the whole array the ranks assemble."""

    world = 2

    def __init__(self, T, split, rank, other):
        self.ranges = [(0, split), (split, T + 1)]
        self.rank = rank
        self.other = other
        self.calls = []

    @property
    def owned_order_range(self):
        return self.ranges[self.rank]

    def gather_columns(self, xp, compact, width, *, name="orders"):
        self.calls.append((name, tuple(compact.shape), int(width)))
        assert xp is torch
        whole = self.other[name]
        out = xp.full_like(whole, complex("nan"))
        for r, (m_lo, m_hi) in enumerate(self.ranges):
            out[..., m_lo:m_hi] = compact if r == self.rank else whole[..., m_lo:m_hi]
        return out


@pytest.mark.parametrize("precision", ["float64", "split16"])
@pytest.mark.parametrize("rank", [0, 1])
def test_order_axis_returns_the_single_card_bits(precision, rank):
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    T = 21
    t = SphericalHarmonicTransform.create(T, precision=precision)
    coeff = torch.as_tensor(red_spectrum(T, 3), device="cuda").to(t.backend.complex_dtype)
    field = t.inverse(coeff)
    spectrum = t.forward(field)
    waist_values = t.contract_to_waist(coeff).take()
    via_waist = t.waist_to_grid(t.contract_to_waist(coeff))
    ex = TwoRankOrderExchange(T, 9, rank, {"analysis_orders": spectrum,
                                           "synthesis_orders": waist_values})
    m_lo, m_hi = ex.owned_order_range
    t.order_exchange = ex
    try:
        got = t.forward(field)
        assert torch.equal(got, spectrum)
        grid = t.inverse(coeff)
        assert torch.equal(grid, via_waist)
        scale = float(via_waist.abs().max())
        tol = 1e-12 if precision == "float64" else 2e-6
        assert float((grid - t._synth("sht_inverse", coeff)).abs().max()) <= tol * scale
    finally:
        t.order_exchange = None
    assert ex.calls == [("analysis_orders", (3, T + 1, m_hi - m_lo), T + 1),
                        ("synthesis_orders", (3, t.grid.nlat, m_hi - m_lo), T + 1)]
    # with the exchange passed explicitly, and with a world of one
    ex.calls.clear()
    assert torch.equal(t.forward_orders(field, ex), spectrum)
    assert len(ex.calls) == 1
    ex.world = 1
    assert torch.equal(t.forward_orders(field, ex), spectrum)
    assert torch.equal(t.inverse_orders(coeff, ex), t.inverse(coeff))
    assert len(ex.calls) == 1
    assert t.owned_order_range == (0, T + 1)


def test_order_exchange_range_is_checked():
    from b200sht import SphericalHarmonicTransform

    t = SphericalHarmonicTransform.create(9, precision="float64")
    ex = TwoRankOrderExchange(9, 4, 0, {})
    ex.ranges = [(3, 3), (3, 10)]
    with pytest.raises(ValueError, match="owned_order_range"):
        t.forward_orders(np.zeros(t.grid.shape), ex)


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_streamed_forms_return_the_resident_bits(precision):
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    T = 31
    t = SphericalHarmonicTransform.create(T, precision=precision)
    rng = np.random.default_rng(T)
    for lead in ((), (3,)):
        field = rng.standard_normal((*lead, *t.grid.shape))
        for chunk in (None, 1, 5, 32):
            assert torch.equal(t.forward_streaming(field, order_chunk=chunk), t.forward(field))
    coeff = red_spectrum(T, 2)
    assert torch.equal(t.inverse_streaming(coeff, order_chunk=4), t.inverse(coeff))
    with pytest.raises(ValueError, match="order_chunk must be >= 1"):
        t.forward_streaming(np.zeros(t.grid.shape), order_chunk=0)
    assert t.streaming_working_bytes(32) == {"recurrence": 0, "analysis": 0, "device": 0,
                                            "scratch": 0}


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_compact_order_contractions(precision):
    """``_contract_orders`` (the reference's rank-local contraction, which its
    multi-card tests call) returns the whole contraction's columns bit for
    bit; ``_analyze`` / ``_synthesize`` are the waist-path transforms."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    T = 21
    t = SphericalHarmonicTransform.create(T, precision=precision)
    coeff = torch.as_tensor(red_spectrum(T, 2), device="cuda").to(t.backend.complex_dtype)
    field = t.inverse(coeff)
    spec = t.contract_waist(t.fourier_waist(field))
    waist = t.contract_to_waist(coeff).take()
    for lo, hi in ((0, 5), (5, 22), (11, 12)):
        got = t._contract_orders(t.fourier_waist(field).take(), t._analysis, lo, hi)
        assert tuple(got.shape) == (2, T + 1, hi - lo) and torch.equal(got, spec[..., lo:hi])
        got = t._contract_orders(coeff, t._basis, lo, hi)
        assert tuple(got.shape) == (2, t.grid.nlat, hi - lo)
        assert torch.equal(got, waist[..., lo:hi])
    with pytest.raises(ValueError, match="non-empty range"):
        t._contract_orders(coeff, t._basis, 4, 4)
    assert torch.equal(t._analyze(field), spec)
    assert torch.equal(t._synthesize(coeff), t.waist_to_grid(t.contract_to_waist(coeff)))
