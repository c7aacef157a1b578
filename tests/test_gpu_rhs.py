"""The fused RHS kernels (sht_rhs_*) against the oracle and the reference's
recorded vertical flux divergence.  Tolerances: float64 1e-13 relative to
the operands' scale, float32 1e-6 (FMA contraction)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-13, torch.float32: 1e-6}
NP = {torch.float64: np.float64, torch.float32: np.float32}


def _close(got, want, dt):
    got = got.cpu().numpy()
    scale = max(float(np.max(np.abs(want))), 1e-300)
    assert float(np.max(np.abs(got - want))) <= TOL[dt] * scale * 4


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("nlon", [16, 18])  # 18: horizontal size not a multiple of 4
def test_momentum_bernoulli(dt, nlon):
    from b200sht.rhs import momentum_bernoulli
    from oracle import rhs as O

    rng = np.random.default_rng(1)
    nlev, nlat = 7, 5
    three = [rng.standard_normal((nlev, nlat, nlon)).astype(NP[dt]) for _ in range(8)]
    two = [rng.standard_normal((nlat, nlon)).astype(NP[dt]) for _ in range(3)]
    zeta, u, v, wu, wv, tv, pg, phi = three
    cor, ge, gn = two
    want = O.momentum_bernoulli(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, NP[dt](287.04))
    dev = lambda a: torch.as_tensor(a, device="cuda")
    got = momentum_bernoulli(dev(zeta), dev(cor), dev(u), dev(v), dev(wu), dev(wv), dev(tv),
                             dev(pg), dev(ge), dev(gn), dev(phi), 287.04)
    for a, b in zip(got, want):
        _close(a, b, dt)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("lead", [(), (3,), (2, 2)])
def test_tracer_flux_and_tendency(dt, lead):
    from b200sht.rhs import scalar_tendency, tracer_flux
    from oracle import rhs as O

    rng = np.random.default_rng(2)
    shape = (6, 4, 12)
    dp = (rng.random(shape) + 0.5).astype(NP[dt])
    u, v, dpt = [rng.standard_normal(shape).astype(NP[dt]) for _ in range(3)]
    s, h, vert = [rng.standard_normal(lead + shape).astype(NP[dt]) for _ in range(3)]
    dev = lambda a: torch.as_tensor(a, device="cuda")
    fl = tracer_flux(dev(dp), dev(s), dev(u), dev(v))
    fx, fy = O.tracer_flux(dp, s, u, v)
    _close(fl[0], fx, dt)
    _close(fl[1], fy, dt)
    _close(scalar_tendency(dev(h), dev(vert), dev(s), dev(dpt), dev(dp)),
           O.scalar_tendency(h, vert, s, dpt, dp), dt)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_elementwise_chains_match_reference(golden, dt):
    """The three elementwise kernels against outputs of the reference's own
    numpy specifications (tests/golden/rhs_elementwise.npz)."""
    from b200sht.rhs import momentum_bernoulli, scalar_tendency, tracer_flux

    tag = "f64" if dt == torch.float64 else "f32"
    g = golden("rhs_elementwise.npz")
    f = {k[: -len(tag) - 1]: g[k] for k in g if k.endswith(tag)}
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    got = momentum_bernoulli(dev(f["zeta"]), dev(f["cor"]), dev(f["u"]), dev(f["v"]), dev(f["wu"]),
                             dev(f["wv"]), dev(f["tv"]), dev(f["pg"]), dev(f["ge"]), dev(f["gn"]),
                             dev(f["phi"]), 287.0528)
    for a, k in zip(got, ("mu", "mv", "bern")):
        _close(a, f[k], dt)
    fx, fy = tracer_flux(dev(f["dp"]), dev(f["s"]), dev(f["u"]), dev(f["v"]))
    _close(fx, f["fx"], dt)
    _close(fy, f["fy"], dt)
    _close(scalar_tendency(dev(f["h"]), dev(f["vert"]), dev(f["s"]), dev(f["dpt"]), dev(f["dp"])),
           f["st"], dt)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_vertical_flux_divergence_matches_reference(golden, dt):
    from b200sht.rhs import vertical_flux_divergence

    tag = "f64" if dt == torch.float64 else "f32"
    g = golden("rhs_vertical_flux.npz")
    dev = lambda a: torch.as_tensor(a, device="cuda")
    got = vertical_flux_divergence(dev(g[f"s_{tag}"]), dev(g[f"w_{tag}"]), dev(g[f"pf_{tag}"]),
                                   dev(g[f"ph_{tag}"]))
    _close(got, g[f"out_{tag}"], dt)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
@pytest.mark.parametrize("nlev", [1, 2, 3, 40])
def test_vertical_flux_divergence_against_oracle(dt, nlev):
    from b200sht.rhs import vertical_flux_divergence
    from oracle import rhs as O

    s, w, pf, ph = O.column_state(nlev, 7, 9, 2, nlev, dtype=NP[dt])
    dev = lambda a: torch.as_tensor(a, device="cuda")
    got = vertical_flux_divergence(dev(s), dev(w), dev(pf), dev(ph))
    _close(got, O.vertical_flux_divergence(s, w, pf, ph), dt)


def test_errors():
    from b200sht.rhs import tracer_flux, vertical_flux_divergence

    x = torch.zeros((4, 3, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="mixed dtypes"):
        tracer_flux(x, x.double(), x, x)
    with pytest.raises(ValueError, match="nlev \\+ 1"):
        vertical_flux_divergence(x, x, x, x)


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_reference_kernel_factories(dt):
    """The reference's ``*_kernel(xp)(...)`` calling forms (fused.py:233-386,
    as dynamics.py calls them): the same bits as the functions, outputs
    written in place when passed."""
    from b200sht import rhs as R

    rng = np.random.default_rng(9)
    nlev, nlat, nlon = 6, 5, 12
    dev = lambda a: torch.as_tensor(a.astype(NP[dt]), device="cuda")
    three = [dev(rng.standard_normal((nlev, nlat, nlon))) for _ in range(8)]
    two = [dev(rng.standard_normal((nlat, nlon))) for _ in range(3)]
    zeta, u, v, wu, wv, tv, pg, phi = three
    cor, ge, gn = two
    want = R.momentum_bernoulli(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, 287.04)
    got = R.momentum_bernoulli_kernel(torch)(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi,
                                             NP[dt](287.04))
    outs = [torch.empty_like(zeta) for _ in range(3)]
    R.momentum_bernoulli_kernel(torch)(zeta, cor, u, v, wu, wv, tv, pg, ge, gn, phi, 287.04,
                                       *outs)
    for a, b, c in zip(got, outs, want):
        assert torch.equal(a, c) and torch.equal(b, c)
    dp = dev(np.abs(rng.standard_normal((nlev, nlat, nlon))) + 1.0)
    s = dev(rng.standard_normal((3, nlev, nlat, nlon)))
    fluxes = torch.empty((2, *s.shape), dtype=dt, device="cuda")
    R.tracer_flux_kernel(torch)(dp, s, u, v, fluxes[0], fluxes[1])
    assert torch.equal(fluxes, R.tracer_flux(dp, s, u, v))
    fx, fy = R.tracer_flux_kernel(torch)(dp, s, u, v)
    assert torch.equal(fx, fluxes[0]) and torch.equal(fy, fluxes[1])
    h, vert = (dev(rng.standard_normal(s.shape)) for _ in range(2))
    dpt = dev(rng.standard_normal((nlev, nlat, nlon)))
    assert torch.equal(R.scalar_tendency_kernel(torch)(h, vert, s, dpt, dp),
                       R.scalar_tendency(h, vert, s, dpt, dp))
    ph = dev(np.cumsum(np.abs(rng.standard_normal((nlev + 1, nlat, nlon))) + 1.0, axis=0))
    pf = torch.sqrt(ph[:-1] * ph[1:]).contiguous()
    w = dev(rng.standard_normal((nlev + 1, nlat, nlon)))
    out = torch.empty_like(s)
    R.vertical_flux_divergence_kernel(torch)(s, w, pf, ph, nlev, nlat * nlon, out)
    assert torch.equal(out, R.vertical_flux_divergence(s, w, pf, ph))
    with pytest.raises(ValueError, match="do not match"):
        R.vertical_flux_divergence_kernel(torch)(s, w, pf, ph, nlev + 1, nlat * nlon, out)
