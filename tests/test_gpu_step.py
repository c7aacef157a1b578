"""The full dycore-step transform set (forward of the scalars, vordiv from the
wind, the Helmholtz solve, wind/gradient/divergence syntheses) against the
oracle's chain of the same calls, its CUDA-graph replay against the eager
run, and the Rossby-Haurwitz wave's energy over repeated steps."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _step(T, precision, nlev, n_scalar, **kw):
    from b200sht import SphericalHarmonicTransform
    from b200sht.semi_implicit import VerticalModeOperator
    from b200sht.step import DycoreTransformStep, rossby_haurwitz_state
    from b200sht.synthetic import seeded_vertical_operator

    b, c = seeded_vertical_operator(nlev)
    op = VerticalModeOperator(b, c)
    f64 = SphericalHarmonicTransform.create(T, precision="float64", **kw)
    state = rossby_haurwitz_state(f64, nlev, n_scalar=n_scalar)
    sht = f64 if precision == "float64" else SphericalHarmonicTransform.create(
        T, precision=precision, **kw)
    return DycoreTransformStep(sht, op, n_scalar=n_scalar), op, state


def _outputs(step):
    np_ = step.t.backend.to_numpy
    return {k: np_(getattr(step, k)).copy() for k in (
        "scalar_coeff", "lnps_coeff", "vorticity", "divergence", "div_solved", "theta_solved",
        "lnps_solved", "u", "v", "grad_theta", "grad_lnps", "div_grid")}


def test_step_matches_oracle_chain_fp64():
    from oracle.dense_sht import DenseSHT, solve_shifted

    T, nlev, ns = 21, 6, 2
    step, op, (scal, lnps, u, v) = _step(T, "float64", nlev, ns)
    step.load(scal, lnps, u, v)
    step.run()
    got = _outputs(step)
    ora = DenseSHT(T)
    sc = ora.forward(scal)
    lp = ora.forward(lnps)
    z, d = ora.vordiv_from_wind(u, v)
    d2, th2, lp2 = solve_shifted(d, sc[0], lp, op.b_matrix, op.c_matrix, op.eigenvalues,
                                 op.eigenvectors, step.tau_s)
    u2, v2 = ora.wind_from_vordiv(z, d2)
    want = {"scalar_coeff": sc, "lnps_coeff": lp, "vorticity": z, "divergence": d,
            "div_solved": d2, "theta_solved": th2, "lnps_solved": lp2, "u": u2, "v": v2,
            "grad_theta": np.stack(ora.gradient(th2)), "grad_lnps": np.stack(ora.gradient(lp2)),
            "div_grid": ora.inverse(d2)}
    for k, w in want.items():
        assert rel_max(got[k], w) < 1e-11, (k, rel_max(got[k], w))


@pytest.mark.parametrize("precision", ["float64", "float32", "split16"])
def test_graph_replay_equals_eager(precision):
    import torch

    step, _, state = _step(62, precision, 8, 5, nlat=94, nlon=192, dealias_factor=1.49)
    step.load(*state)
    step.prepare()
    step.run()
    torch.cuda.synchronize()
    eager = _outputs(step)
    step.load(*state)
    step.capture()
    step.load(*state)
    step.replay(1)
    torch.cuda.synchronize()
    step.t.check_device()
    graphed = _outputs(step)
    for k in eager:
        assert np.array_equal(eager[k], graphed[k]), k
    # Replays start from the wind the previous replay wrote; reloading the
    # state starts over.
    step.replay(1)
    step.load(*state)
    step.replay(1)
    torch.cuda.synchronize()
    assert np.array_equal(_outputs(step)["u"], eager["u"])


@pytest.mark.parametrize("precision,bar", [("float64", 1e-11), ("split16", 2e-5)])
def test_rossby_haurwitz_wave_energy_over_steps(precision, bar):
    """Vorticity energy of the wave (n = 5, m = 4) and of the solid-body part
    (n = 1, m = 0) after 25 graph-replayed steps, against the first step."""
    import torch
    from b200sht.step import wave_energy

    T = 42
    step, _, state = _step(T, precision, 4, 1)
    step.load(*state)
    step.capture()
    step.load(*state)
    step.replay(1)
    torch.cuda.synchronize()
    np_ = step.t.backend.to_numpy
    z0 = np_(step.vorticity).copy()
    step.replay(25)
    torch.cuda.synchronize()
    step.t.check_device()
    z1 = np_(step.vorticity)
    for n, m in ((5, 4), (1, 0)):
        drift = wave_energy(z1, n, m, T) / wave_energy(z0, n, m, T) - 1.0
        assert abs(drift) < bar, (n, m, drift)
