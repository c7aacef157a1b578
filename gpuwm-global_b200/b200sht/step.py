"""The transform calls of one semi-implicit dycore step, recorded as one CUDA graph.

Per 300 s step the reference's dycore (src/arwen_global/dynamics.py:1178-1717,
semilag/step.py:1412-1673, semi_implicit.py:921-953) analyses its scalar
fields, analyses vorticity and divergence from the wind, solves the per-degree
semi-implicit Helmholtz problem, and synthesises the wind, the temperature
and surface-pressure gradients and the solved divergence.  ``DycoreTransformStep``
holds every buffer of that call set on the device and issues it as:

1. ``forward``: ``n_scalar x nlev`` scalar planes (temperature first) and ln ps;
2. ``vordiv_from_wind``: (u, v) -> (zeta, D), ``nlev`` levels;
3. ``sht_helmholtz_synthesis``: (D, theta, ln ps) -> (D', theta', ln ps') and
   the grid divergence, the solve writing D' straight into the synthesis
   operand (the Helmholtz solve fused into the synthesis prologue);
4. ``wind_from_vordiv``: (zeta, D') -> (u, v), written back into the input wind;
5. ``gradient``: of theta' (``nlev`` planes) and ln ps' (one plane).

Step 4 overwrites the wind the next step starts from, so replaying the graph
iterates the step.  Nothing in it allocates, copies from the host or
synchronises once the plan's scratch and tile lists exist (``prepare``), so
``capture`` records the whole set in one ``torch.cuda.CUDAGraph``.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .semi_implicit import VerticalModeOperator, VerticalModeSemiImplicit
from .transform import SphericalHarmonicTransform, _ptr, _stream


class DycoreTransformStep:
    def __init__(self, transform: SphericalHarmonicTransform, vertical: VerticalModeOperator,
                 *, n_scalar: int = 5, dt_s: float = 300.0, alpha: float = 0.5):
        if n_scalar < 1:
            raise ValueError("n_scalar must be >= 1 (the first scalar is the temperature)")
        self.t = transform
        self.vertical = vertical
        self.solver = VerticalModeSemiImplicit()
        self.nlev = vertical.nlev
        self.n_scalar = int(n_scalar)
        self.tau_s = float(alpha) * float(dt_s)
        t, L = transform, vertical.nlev
        g, s = t._empty_grid, t._empty_spec
        # Inputs (grid).
        self.scalars = g((self.n_scalar, L))
        self.lnps = g(())
        self.u = g((L,))
        self.v = g((L,))
        # Spectral intermediates and outputs.
        self.scalar_coeff = s((self.n_scalar, L))
        self.lnps_coeff = s(())
        self.vorticity = s((L,))
        self.divergence = s((L,))
        self.div_solved = s((L,))
        self.theta_solved = s((L,))
        self.lnps_solved = s(())
        # Grid outputs.
        self.grad_theta = g((2, L))
        self.grad_lnps = g((2,))
        self.div_grid = g((L,))
        self.graph = None

    # ------------------------------------------------------------------ set-up
    def load(self, scalars, lnps, u, v) -> None:
        """Copy a state into the step's input buffers (outside any graph)."""
        for dst, src in ((self.scalars, scalars), (self.lnps, lnps), (self.u, u), (self.v, v)):
            dst.copy_(torch.as_tensor(src).to(dst.device, dst.dtype))

    def prepare(self) -> None:
        """Grow the plan's scratch to the largest call, upload the vertical
        operator and build every per-size work list, by running the step
        once (the inputs are restored afterwards)."""
        saved = [x.clone() for x in (self.scalars, self.lnps, self.u, self.v)]
        self.vertical.device_handle(self.t)
        self.run()
        torch.cuda.current_stream().synchronize()
        for dst, src in zip((self.scalars, self.lnps, self.u, self.v), saved):
            dst.copy_(src)
        torch.cuda.current_stream().synchronize()

    # ------------------------------------------------------------------- step
    def run(self) -> None:
        """Issue the step's calls on the current stream (eager)."""
        t, L, h, st = self.t, self.nlev, self.t.plan.handle, _stream()
        _lib.call("sht_forward", h, _ptr(self.scalars), self.n_scalar * L,
                  _ptr(self.scalar_coeff), st)
        _lib.call("sht_forward", h, _ptr(self.lnps), 1, _ptr(self.lnps_coeff), st)
        _lib.call("sht_vordiv_from_wind", h, _ptr(self.u), _ptr(self.v), L, _ptr(self.vorticity),
                  _ptr(self.divergence), st)
        self.solver.solve_and_synthesize_into(t, self.vertical, self.tau_s, self.divergence,
                                              self.scalar_coeff[0], self.lnps_coeff,
                                              self.div_solved, self.theta_solved,
                                              self.lnps_solved, self.div_grid)
        _lib.call("sht_wind_from_vordiv", h, _ptr(self.vorticity), _ptr(self.div_solved), L,
                  _ptr(self.u), _ptr(self.v), st)
        _lib.call("sht_gradient", h, _ptr(self.theta_solved), L, _ptr(self.grad_theta[0]),
                  _ptr(self.grad_theta[1]), st)
        _lib.call("sht_gradient", h, _ptr(self.lnps_solved), 1, _ptr(self.grad_lnps[0]),
                  _ptr(self.grad_lnps[1]), st)

    def capture(self) -> torch.cuda.CUDAGraph:
        """Record ``run`` in a CUDA graph (``prepare`` first)."""
        self.prepare()
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side), torch.cuda.graph(graph, stream=side):
            self.run()
        torch.cuda.current_stream().wait_stream(side)
        self.graph = graph
        return graph

    def replay(self, steps: int = 1) -> None:
        if self.graph is None:
            raise RuntimeError("capture() the step first")
        for _ in range(int(steps)):
            self.graph.replay()

    # ------------------------------------------------------------ diagnostics
    def transforms_per_step(self) -> dict:
        """Planes through each transform kind per step."""
        L = self.nlev
        return {"scalar_analysis": self.n_scalar * L + 1, "vordiv_analysis": L,
                "wind_synthesis": L, "gradient_synthesis": L + 1, "scalar_synthesis": L}


def wave_energy(vorticity: np.ndarray, n: int, m: int, truncation: int) -> float:
    """Spectral energy ``w_m |zeta_nm|^2`` of one (n, m) vorticity component
    summed over levels (``w_0 = 1``, ``w_m>0 = 2``)."""
    z = np.asarray(vorticity).reshape(-1, truncation + 1, truncation + 1)
    w = 1.0 if m == 0 else 2.0
    return float(w * np.sum(np.abs(z[:, n, m]) ** 2))


def rossby_haurwitz_state(transform: SphericalHarmonicTransform, nlev: int, *,
                          noise: float = 0.01, n_scalar: int = 5, seed: int | None = None):
    """Initial state of the full-step workload: the wavenumber-4
    Rossby-Haurwitz wind (omega = K = 7.848e-6 1/s) on every level plus a
    seeded red-spectrum wind at ``noise`` of its RMS, red-spectrum scalars
    and ln ps.  Host numpy arrays ``(scalars, lnps, u, v)``; the noise wind and
    the scalars are synthesised by ``transform`` (use a float64 transform)."""
    from .synthetic import CONTROL_SEED, red_spectrum, rossby_haurwitz_wind
    from .vector import VorticityDivergenceOperator

    seed = CONTROL_SEED if seed is None else int(seed)
    t = transform
    T = t.truncation
    to_np = t.backend.to_numpy
    u0, v0 = rossby_haurwitz_wind(t.grid.sin_lat, t.grid.nlon, radius_m=t.grid.radius_m)
    un, vn = (to_np(x) for x in VorticityDivergenceOperator(t).wind_from_vordiv(
        red_spectrum(T, nlev, seed + 11), red_spectrum(T, nlev, seed + 12)))
    rms0 = float(np.sqrt(np.mean(u0 ** 2 + v0 ** 2)))
    rmsn = float(np.sqrt(np.mean(un ** 2 + vn ** 2)))
    k = noise * rms0 / max(rmsn, 1e-300)
    u = u0[None] + k * un
    v = v0[None] + k * vn
    scal = to_np(t.inverse(red_spectrum(T, n_scalar * nlev, seed + 13))).reshape(
        n_scalar, nlev, *t.grid.shape)
    lnps = to_np(t.inverse(red_spectrum(T, 1, seed + 14)[0]))
    return scal, lnps, u, v
