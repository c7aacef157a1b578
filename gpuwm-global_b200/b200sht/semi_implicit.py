"""Per-degree semi-implicit maps in the vertical-mode basis.

Mirror of the reference's ``VerticalModeSemiImplicit``
(src/arwen_global/semi_implicit.py:697-953): ``solve_shifted`` (the IMEX stage
solve), ``apply`` (the off-centred Crank-Nicolson step), ``half_apply`` (its
square root, applied before and after the explicit step: ``pre_apply`` /
``post_apply``).  Each is one library call (``sht_semi_implicit_map``) that
applies the per-degree operators modally on the device.  The third argument
is the reference's vertical coordinate (any object with ``nlev``,
``a_half_pa``, ``b_half`` and ``hydrostatic_geopotential``; the operator is
built from it once per reference state, as the reference's
``vertical_structure_operator`` does) or a ready ``VerticalModeOperator``.

The operator build (``VerticalModeOperator.from_coordinate``) is host float64
numpy, as in the reference (``VerticalStructureOperator._build``,
semi_implicit.py:421-577): B (nlev x nlev+1) and C (nlev+1 x nlev) of the
linear gravity-wave operator about an isothermal reference, the modes of
M = -B C, and the modes of the thermodynamic block C B for the half maps.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from dataclasses import dataclass
from typing import NamedTuple

import numpy as np
import torch

from . import _lib
from .transform import SphericalHarmonicTransform, _ptr, _stream

#: The reference's physical constants (src/arwen_global/spectral/constants.py).
DRY_AIR_GAS_CONSTANT = 287.0
DRY_AIR_CP = 1004.0
KAPPA = DRY_AIR_GAS_CONSTANT / DRY_AIR_CP
REFERENCE_PRESSURE_PA = 100_000.0
GRAVITY_M_S2 = 9.80616


def _real_modes(matrix, what):
    values, vectors = np.linalg.eig(matrix)
    if np.max(np.abs(values.imag)) > 1.0e-9 * np.max(np.abs(values.real)):
        raise ValueError(f"{what} has complex eigenvalues: the reference state does not "
                         "define real gravity-wave modes")
    return values.real, vectors.real


class VerticalModeOperator:
    """``B`` (nlev x nlev+1), ``C`` (nlev+1 x nlev), the modes of
    ``M = -B C`` (eigenvalues descending, real and positive) and of the
    thermodynamic block ``C B`` (eigenvalues <= 0, one null mode)."""

    def __init__(self, b_matrix, c_matrix, eigenvalues=None, eigenvectors=None,
                 x_eigenvalues=None, x_eigenvectors=None):
        b = np.ascontiguousarray(b_matrix, dtype=np.float64)
        c = np.ascontiguousarray(c_matrix, dtype=np.float64)
        nlev = b.shape[0]
        if b.shape != (nlev, nlev + 1) or c.shape != (nlev + 1, nlev):
            raise ValueError(f"B must be (nlev, nlev+1) and C (nlev+1, nlev), got {b.shape}, {c.shape}")
        if eigenvalues is None:
            values, vectors = _real_modes(-b @ c, "vertical-structure matrix")
            if np.min(values) <= 0.0:
                raise ValueError("vertical-structure matrix has a nonpositive eigenvalue: a mode of "
                                 "the reference state would grow instead of oscillate")
            order = np.argsort(-values)
            eigenvalues = values[order]
            eigenvectors = vectors[:, order]
        if x_eigenvalues is None:
            # C B shares the nonzero spectrum of B C and adds the null mode
            # of B at zero (the reference's reading, semi_implicit.py:551-565).
            xv, xw = _real_modes(c @ b, "thermodynamic block of the vertical-structure operator")
            xv[np.abs(xv) <= 1.0e-9 * np.max(np.abs(xv))] = 0.0
            if np.max(xv) > 0.0:
                raise ValueError("thermodynamic block of the vertical-structure operator has a "
                                 "positive eigenvalue: a mode of the reference state would grow "
                                 "instead of oscillate")
            x_eigenvalues, x_eigenvectors = xv, xw
        self.b_matrix = b
        self.c_matrix = c
        self.eigenvalues = np.ascontiguousarray(eigenvalues, dtype=np.float64)
        self.eigenvectors = np.ascontiguousarray(eigenvectors, dtype=np.float64)
        self.eigenvectors_inv = np.ascontiguousarray(np.linalg.inv(self.eigenvectors))
        self.x_eigenvalues = np.ascontiguousarray(x_eigenvalues, dtype=np.float64)
        self.x_eigenvectors = np.ascontiguousarray(x_eigenvectors, dtype=np.float64)
        self.x_eigenvectors_inv = np.ascontiguousarray(np.linalg.inv(self.x_eigenvectors))
        # The reference state (set by from_coordinate; None for an operator
        # built from ready matrices) and the modes as the reference reports
        # them (semi_implicit.py:551-570).
        self.reference_temperature_k = None
        self.reference_surface_pressure_pa = None
        self.phase_speeds_m_s = np.sqrt(self.eigenvalues)
        self.equivalent_depths_m = self.eigenvalues / GRAVITY_M_S2

    @property
    def fastest_mode_m_s(self) -> float:
        return float(self.phase_speeds_m_s[0])

    def describe(self) -> dict:
        return {
            "reference_temperature_k": self.reference_temperature_k,
            "reference_surface_pressure_pa": self.reference_surface_pressure_pa,
            "nlev": self.nlev,
            "phase_speeds_m_s": [float(v) for v in self.phase_speeds_m_s],
            "equivalent_depths_m": [float(v) for v in self.equivalent_depths_m],
        }

    @classmethod
    def from_coordinate(cls, vertical, reference_temperature_k: float,
                        reference_surface_pressure_pa: float, *,
                        gas_constant: float = DRY_AIR_GAS_CONSTANT) -> "VerticalModeOperator":
        """The linear gravity-wave operator of a hybrid stack about an
        isothermal reference (semi_implicit.py:421-577), built from the
        coordinate's half-level A/B and its own hydrostatic integration.

        Rows of B: the pressure-gradient response of each level's divergence
        tendency to theta (through the geopotential, times the Exner factor)
        and to ln ps.  Rows of C: minus the theta tendency per unit
        divergence (continuity, the interface pressure velocity and the
        flux-form vertical advection of the reference theta through a
        limited interface reconstruction), and minus the layer mass weights
        (the ln ps tendency)."""
        nlev = int(vertical.nlev)
        t_ref = float(reference_temperature_k)
        ps = float(reference_surface_pressure_pa)
        rgas = float(gas_constant)
        a_half = np.asarray(vertical.a_half_pa, dtype=np.float64)
        b_half = np.asarray(vertical.b_half, dtype=np.float64)
        p_half = a_half + b_half * ps
        p_full = np.sqrt(p_half[:-1] * p_half[1:])
        dp = np.diff(p_half)
        db = np.diff(b_half)
        exner = (p_full / REFERENCE_PRESSURE_PA) ** KAPPA
        theta0 = t_ref / exner
        dlnp_dlnps = 0.5 * (b_half[:-1] / p_half[:-1] + b_half[1:] / p_half[1:]) * ps
        # Geopotential per unit virtual temperature at each level: the
        # coordinate's own integration is linear in Tv at fixed pressure.
        geo = np.empty((nlev, nlev))
        for j in range(nlev):
            unit = np.zeros((nlev, 1, 1))
            unit[j] = 1.0
            geo[:, j] = vertical.hydrostatic_geopotential(
                unit, np.zeros((1, 1)), p_half[:, None, None], gas_constant=rgas)[:, 0, 0]
        # Interface theta0: the limited one-sided reconstructions from the
        # layers above and below, each clipped to the two layers, averaged.
        slope = np.zeros(nlev)
        up = (theta0[1:-1] - theta0[:-2]) / (p_full[1:-1] - p_full[:-2])
        down = (theta0[2:] - theta0[1:-1]) / (p_full[2:] - p_full[1:-1])
        same = up * down > 0.0
        slope[1:-1] = np.where(same, 2.0 * (up * down) / np.where(same, up + down, 1.0), 0.0)
        lo = np.minimum(theta0[:-1], theta0[1:])
        hi = np.maximum(theta0[:-1], theta0[1:])
        from_above = np.clip(theta0[:-1] + slope[:-1] * (p_half[1:nlev] - p_full[:-1]), lo, hi)
        from_below = np.clip(theta0[1:] + slope[1:] * (p_half[1:nlev] - p_full[1:]), lo, hi)
        face = np.zeros(nlev + 1)
        face[1:nlev] = 0.5 * (from_above + from_below)
        # Theta tendency per unit divergence at level j (column j), by the
        # continuity equation of a unit mass-flux divergence dp_j at level j.
        gamma = np.empty((nlev, nlev))
        for j in range(nlev):
            mfd = np.zeros(nlev)
            mfd[j] = dp[j]
            dps_dt = -dp[j]
            ddp_dt = db * dps_dt
            omega = np.zeros(nlev + 1)
            for k in range(nlev):
                omega[k + 1] = omega[k] - ddp_dt[k] - mfd[k]
            omega[nlev] = 0.0
            flux = omega * face
            dtheta = (-(mfd * theta0) - (flux[1:] - flux[:-1]) - theta0 * ddp_dt) / dp
            gamma[:, j] = -dtheta
        b = np.empty((nlev, nlev + 1))
        b[:, :nlev] = geo * exner[None, :]
        b[:, nlev] = KAPPA * t_ref * (geo @ dlnp_dlnps) + rgas * t_ref
        c = np.empty((nlev + 1, nlev))
        c[:nlev] = -gamma
        c[nlev] = -(dp / ps)
        op = cls(b, c)
        op.reference_temperature_k = t_ref
        op.reference_surface_pressure_pa = ps
        return op

    @property
    def nlev(self) -> int:
        return int(self.b_matrix.shape[0])

    def device_handle(self, transform: SphericalHarmonicTransform) -> "DeviceVerticalOperator":
        """The operator uploaded for ``transform``'s device and precision
        (created on first use and kept, like the reference's per-run
        ``VerticalStructureOperator``)."""
        key = (str(transform.backend.device), transform.precision)
        cache = self.__dict__.setdefault("_device_handles", {})
        if key not in cache:
            cache[key] = DeviceVerticalOperator(transform, self)
        return cache[key]


class DeviceVerticalOperator:
    """One ``sht_vertical`` handle: B, C and both modal bases resident on the
    device, so that the maps copy and allocate nothing per call."""

    def __init__(self, transform: SphericalHarmonicTransform, op: VerticalModeOperator):
        self._lib = _lib.load()
        dp = ctypes.POINTER(ctypes.c_double)
        handle = ctypes.c_void_p()
        with torch.cuda.device(transform.backend.device):
            _lib.check(self._lib.sht_vertical_create_modes(
                transform.plan.handle, op.nlev, op.b_matrix.ctypes.data_as(dp),
                op.c_matrix.ctypes.data_as(dp), op.eigenvectors.ctypes.data_as(dp),
                op.eigenvectors_inv.ctypes.data_as(dp), op.eigenvalues.ctypes.data_as(dp),
                op.x_eigenvectors.ctypes.data_as(dp), op.x_eigenvectors_inv.ctypes.data_as(dp),
                op.x_eigenvalues.ctypes.data_as(dp), ctypes.byref(handle)))
        self.handle = handle
        self.nlev = op.nlev

    def metric(self) -> float:
        """max |D' - D| of the last map (one device read)."""
        out = ctypes.c_double(0.0)
        _lib.call("sht_semi_implicit_metric", self.handle, ctypes.byref(out), _stream())
        return float(out.value)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.sht_vertical_destroy(h)
            except Exception:
                pass
            self.handle = None


#: Operators built from a coordinate, one per (A, B, T_ref, ps_ref), like the
#: reference's module-level cache (semi_implicit.py:666-694).
_OPERATORS: dict = {}


def vertical_structure_operator(vertical, reference_temperature_k: float,
                                reference_surface_pressure_pa: float) -> VerticalModeOperator:
    key = (np.asarray(vertical.a_half_pa, dtype=np.float64).tobytes(),
           np.asarray(vertical.b_half, dtype=np.float64).tobytes(),
           float(reference_temperature_k), float(reference_surface_pressure_pa))
    op = _OPERATORS.get(key)
    if op is None:
        op = VerticalModeOperator.from_coordinate(vertical, reference_temperature_k,
                                                  reference_surface_pressure_pa)
        _OPERATORS[key] = op
    return op


@dataclass
class SpectralState:
    """The spectral fields the maps read and write."""
    vorticity: object
    divergence: object
    theta: object
    log_surface_pressure: object
    qv: object = None


_METRIC = "semi_implicit_max_divergence_increment_s1"


class LinearTendencies(NamedTuple):
    """The weighted linear triple the explicit right-hand side must not
    integrate (semi_implicit.py:205-215): ``(nlev, T+1, T+1)`` divergence
    and theta tendencies and the ``(T+1, T+1)`` ln ps tendency."""

    divergence: object
    theta: object
    log_surface_pressure: object


@dataclass(frozen=True)
class VerticalModeSemiImplicit:
    """Every vertical gravity-wave mode implicit; the reference's fields,
    defaults and refusals (semi_implicit.py:697-766)."""

    enabled: bool = True
    reference_temperature_k: float = 320.0
    reference_surface_pressure_pa: float = 1.0e5
    off_centring_weight: float = 0.5
    divergence_weight: float = 1.0

    def __post_init__(self):
        if not math.isfinite(self.reference_temperature_k) or not (
                150.0 <= self.reference_temperature_k <= 400.0):
            raise ValueError("reference_temperature_k must lie in 150..400 K: the isothermal "
                             "reference sets every implicit mode speed (sqrt(R T / (1 - kappa)) "
                             "for the external mode)")
        if not math.isfinite(self.reference_surface_pressure_pa) or not (
                30_000.0 <= self.reference_surface_pressure_pa <= 120_000.0):
            raise ValueError("reference_surface_pressure_pa must lie in the 30000..120000 Pa "
                             "research bounds the hybrid stack is evaluated at")
        if not math.isfinite(self.off_centring_weight) or not (
                0.5 <= self.off_centring_weight <= 1.0):
            raise ValueError("off_centring_weight must lie in [0.5, 1]: below 0.5 the implicit "
                             "step amplifies every gravity-wave mode it treats "
                             "(|(1 + (1-a) z)/(1 - a z)| > 1 on the imaginary axis)")
        if not math.isfinite(self.divergence_weight) or not 0.0 <= self.divergence_weight <= 1.0:
            raise ValueError("divergence_weight must lie in [0,1]")

    @property
    def active(self) -> bool:
        return self.enabled and self.divergence_weight > 0.0

    @property
    def scheme(self) -> str:
        return "vertical_modes"

    def operator(self, vertical) -> VerticalModeOperator:
        """The operator of ``vertical`` (a coordinate, or an operator itself)."""
        if isinstance(vertical, VerticalModeOperator):
            return vertical
        return vertical_structure_operator(vertical, self.reference_temperature_k,
                                           self.reference_surface_pressure_pa)

    def explicit_wave_speed_m_s(self, vertical) -> float:
        """The fastest mode speed times the fraction left explicit
        (semi_implicit.py:776-781)."""
        fastest = self.operator(vertical).fastest_mode_m_s
        if self.active:
            return (1.0 - self.divergence_weight) * fastest
        return fastest

    def describe(self, vertical) -> dict:
        """semi_implicit.py:783-790."""
        return {
            "scheme": self.scheme,
            "enabled": bool(self.enabled),
            "off_centring_weight": float(self.off_centring_weight),
            "weight": float(self.divergence_weight),
            **self.operator(vertical).describe(),
        }

    def linear_tendencies(self, state, transform, vertical):
        """``w L y``: the divergence, theta and ln ps tendencies of the
        weighted linear operator at the state, ``D_t = w k^2 (B x)`` and
        ``x_t = w (C D)`` with ``x = (theta, ln ps)``, projected
        (semi_implicit.py:796-813): one library call
        (``SHT_SEMI_LINEAR_TENDENCIES``).  None when inactive."""
        if not self.active:
            return None
        (d, th, lp), _ = self._map(transform, self.operator(vertical),
                                   _lib.SHT_SEMI_LINEAR_TENDENCIES, self.divergence_weight,
                                   state.divergence, state.theta, state.log_surface_pressure)
        return LinearTendencies(d, th, lp)

    # ----------------------------------------------------------- arrays
    def _map(self, transform, operator, mode, dt_w, divergence, theta, lnps, outs=None):
        t = transform
        d = t._spec_in(divergence)
        th = t._spec_in(theta)
        lp = t._spec_in(lnps)
        nlev = operator.nlev
        if d.shape[0] != nlev or th.shape[0] != nlev or d.dim() != 3 or th.dim() != 3 or lp.dim() != 2:
            raise ValueError("divergence/theta must be (nlev, T+1, T+1) and lnps (T+1, T+1)")
        if outs is None:
            outs = (torch.empty_like(d), torch.empty_like(th), torch.empty_like(lp))
        handle = operator.device_handle(t)
        _lib.call("sht_semi_implicit_map", t.plan.handle, handle.handle, int(mode), float(dt_w),
                  float(self.off_centring_weight), _ptr(d), _ptr(th), _ptr(lp), _ptr(outs[0]),
                  _ptr(outs[1]), _ptr(outs[2]), _stream())
        return outs, handle

    def solve_arrays(self, transform: SphericalHarmonicTransform, operator, tau_s: float,
                     divergence, theta, lnps):
        """``(D, theta, ln ps)`` after ``(I - tau w L) y = r``; inputs are
        ``(nlev, T+1, T+1)``, ``(nlev, T+1, T+1)``, ``(T+1, T+1)`` complex."""
        outs, _ = self._map(transform, self.operator(operator), _lib.SHT_SEMI_SOLVE_SHIFTED,
                            float(tau_s) * self.divergence_weight, divergence, theta, lnps)
        return outs

    def solve_into(self, transform, operator, tau_s, divergence, theta, lnps, out_divergence,
                   out_theta, out_lnps) -> None:
        """``solve_arrays`` on caller-owned device arrays (outputs may alias
        inputs): one library call with the operator kept on the device, so no
        allocation, host copy or synchronisation happens here once the
        operator has been uploaded."""
        handle = self.operator(operator).device_handle(transform)
        _lib.call("sht_helmholtz_apply", transform.plan.handle, handle.handle,
                  float(tau_s) * self.divergence_weight, _ptr(divergence), _ptr(theta),
                  _ptr(lnps), _ptr(out_divergence), _ptr(out_theta), _ptr(out_lnps), _stream())

    def solve_and_synthesize_into(self, transform, operator, tau_s, divergence, theta, lnps,
                                  out_divergence, out_theta, out_lnps, divergence_grid) -> None:
        """``solve_into`` with the synthesis of the solved divergence fused
        onto it (``sht_helmholtz_synthesis``): ``divergence_grid`` receives
        ``transform.inverse(out_divergence)``."""
        handle = self.operator(operator).device_handle(transform)
        _lib.call("sht_helmholtz_synthesis", transform.plan.handle, handle.handle,
                  float(tau_s) * self.divergence_weight, _ptr(divergence), _ptr(theta),
                  _ptr(lnps), _ptr(out_divergence), _ptr(out_theta), _ptr(out_lnps),
                  _ptr(divergence_grid), _stream())

    # ------------------------------------------------------------ states
    @staticmethod
    def _rebuild(state, d, th, lp):
        if dataclasses.is_dataclass(state):
            return dataclasses.replace(state, divergence=d, theta=th, log_surface_pressure=lp)
        return state.with_fields((state.vorticity, d, th, lp, state.qv, state.qc, state.qr,
                                  state.qi, state.qs, state.qg))

    def _state_map(self, mode, state, transform, vertical, dt_s, metric=True):
        op = self.operator(vertical)
        (d, th, lp), handle = self._map(transform, op, mode, float(dt_s) * self.divergence_weight,
                                        state.divergence, state.theta, state.log_surface_pressure)
        out = self._rebuild(state, d, th, lp)
        return out, ({_METRIC: handle.metric()} if metric else None)

    def solve_shifted(self, state, transform, vertical, tau_s):
        """The IMEX stage solve ``(I - tau w L) y = r`` (semi_implicit.py:921-953);
        inactive: identity."""
        if not self.active:
            return state
        return self._state_map(_lib.SHT_SEMI_SOLVE_SHIFTED, state, transform, vertical, tau_s,
                               metric=False)[0]

    def apply(self, state, transform, vertical, dt_s):
        """The off-centred Crank-Nicolson step of the subtracted operator over
        ``dt`` (semi_implicit.py:887-919); returns ``(state, metrics)``."""
        if not self.active:
            return state, {_METRIC: 0.0}
        return self._state_map(_lib.SHT_SEMI_APPLY, state, transform, vertical, dt_s)

    def half_apply(self, state, transform, vertical, dt_s):
        """The square root of ``apply``'s map (semi_implicit.py:845-877): applied
        before and after the explicit step it composes to ``apply``."""
        if not self.active:
            return state, {_METRIC: 0.0}
        return self._state_map(_lib.SHT_SEMI_HALF_APPLY, state, transform, vertical, dt_s)

    def pre_apply(self, state, transform, vertical, dt_s):
        """The half map before the explicit step (symmetric split)."""
        return self.half_apply(state, transform, vertical, dt_s)

    def post_apply(self, state, transform, vertical, dt_s):
        """The half map after the explicit step (symmetric split)."""
        return self.half_apply(state, transform, vertical, dt_s)
