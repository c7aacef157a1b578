"""Per-degree semi-implicit Helmholtz solve in the vertical-mode basis.

Mirror of the reference's ``VerticalModeSemiImplicit.solve_shifted``
(src/arwen_global/semi_implicit.py:921-953) and of the modal part of
``VerticalStructureOperator`` (semi_implicit.py:391-609): the structure matrix
``M = -B C`` is eigen-decomposed in float64 on the host (the reference does
the same, semi_implicit.py:505), and the device kernel applies
``V diag(1/(1 + tau^2 k_n^2 lambda)) V^-1`` per coefficient.  The hybrid
coordinate that produces ``B`` and ``C`` in the reference is outside this
engine: callers pass the two matrices (or a seeded synthetic stack).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .transform import SphericalHarmonicTransform, _ptr, _stream


class VerticalModeOperator:
    """``B`` (nlev x nlev+1), ``C`` (nlev+1 x nlev) and the modes of
    ``M = -B C`` (eigenvalues descending, real and positive)."""

    def __init__(self, b_matrix, c_matrix, eigenvalues=None, eigenvectors=None):
        b = np.ascontiguousarray(b_matrix, dtype=np.float64)
        c = np.ascontiguousarray(c_matrix, dtype=np.float64)
        nlev = b.shape[0]
        if b.shape != (nlev, nlev + 1) or c.shape != (nlev + 1, nlev):
            raise ValueError(f"B must be (nlev, nlev+1) and C (nlev+1, nlev), got {b.shape}, {c.shape}")
        if eigenvalues is None:
            structure = -b @ c
            values, vectors = np.linalg.eig(structure)
            if np.max(np.abs(values.imag)) > 1.0e-9 * np.max(np.abs(values.real)):
                raise ValueError("vertical-structure matrix has complex eigenvalues: the reference "
                                 "state does not define real gravity-wave modes")
            if np.min(values.real) <= 0.0:
                raise ValueError("vertical-structure matrix has a nonpositive eigenvalue: a mode of "
                                 "the reference state would grow instead of oscillate")
            order = np.argsort(-values.real)
            eigenvalues = values.real[order]
            eigenvectors = vectors.real[:, order]
        self.b_matrix = b
        self.c_matrix = c
        self.eigenvalues = np.ascontiguousarray(eigenvalues, dtype=np.float64)
        self.eigenvectors = np.ascontiguousarray(eigenvectors, dtype=np.float64)
        self.eigenvectors_inv = np.ascontiguousarray(np.linalg.inv(self.eigenvectors))

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
    """One ``sht_vertical`` handle: B, C and the modal basis resident on the
    device, so that ``sht_helmholtz_apply`` copies and allocates nothing."""

    def __init__(self, transform: SphericalHarmonicTransform, op: VerticalModeOperator):
        self._lib = _lib.load()
        dp = ctypes.POINTER(ctypes.c_double)
        handle = ctypes.c_void_p()
        with torch.cuda.device(transform.backend.device):
            _lib.check(self._lib.sht_vertical_create(
                transform.plan.handle, op.nlev, op.b_matrix.ctypes.data_as(dp),
                op.c_matrix.ctypes.data_as(dp), op.eigenvectors.ctypes.data_as(dp),
                op.eigenvectors_inv.ctypes.data_as(dp), op.eigenvalues.ctypes.data_as(dp),
                ctypes.byref(handle)))
        self.handle = handle
        self.nlev = op.nlev

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.sht_vertical_destroy(h)
            except Exception:
                pass
            self.handle = None


@dataclass
class SpectralState:
    """The spectral fields the stage solve reads and writes."""
    vorticity: object
    divergence: object
    theta: object
    log_surface_pressure: object
    qv: object = None


@dataclass(frozen=True)
class VerticalModeSemiImplicit:
    enabled: bool = True
    divergence_weight: float = 1.0

    def __post_init__(self):
        if not math.isfinite(self.divergence_weight) or not 0.0 <= self.divergence_weight <= 1.0:
            raise ValueError("divergence_weight must lie in [0,1]")

    @property
    def active(self) -> bool:
        return self.enabled and self.divergence_weight > 0.0

    def solve_arrays(self, transform: SphericalHarmonicTransform, operator: VerticalModeOperator,
                     tau_s: float, divergence, theta, lnps):
        """``(D, theta, ln ps)`` after ``(I - tau w L) y = r``; inputs are
        ``(nlev, T+1, T+1)``, ``(nlev, T+1, T+1)``, ``(T+1, T+1)`` complex."""
        t = transform
        d = t._spec_in(divergence)
        th = t._spec_in(theta)
        lp = t._spec_in(lnps)
        nlev = operator.nlev
        if d.shape[0] != nlev or th.shape[0] != nlev or d.dim() != 3 or th.dim() != 3 or lp.dim() != 2:
            raise ValueError("divergence/theta must be (nlev, T+1, T+1) and lnps (T+1, T+1)")
        od, oth, olp = torch.empty_like(d), torch.empty_like(th), torch.empty_like(lp)
        self.solve_into(t, operator, tau_s, d, th, lp, od, oth, olp)
        return od, oth, olp

    def solve_into(self, transform, operator, tau_s, divergence, theta, lnps, out_divergence,
                   out_theta, out_lnps) -> None:
        """``solve_arrays`` on caller-owned device arrays (outputs may alias
        inputs): one ``sht_helmholtz_apply`` with the operator kept on the
        device, so no allocation, host copy or synchronisation happens here
        once the operator has been uploaded."""
        handle = operator.device_handle(transform)
        _lib.call("sht_helmholtz_apply", transform.plan.handle, handle.handle,
                  float(tau_s) * self.divergence_weight, _ptr(divergence), _ptr(theta),
                  _ptr(lnps), _ptr(out_divergence), _ptr(out_theta), _ptr(out_lnps), _stream())

    def solve_shifted(self, state, transform, operator, tau_s):
        """The IMEX stage solve (semi_implicit.py:921-953); inactive: identity."""
        if not self.active:
            return state
        d, th, lp = self.solve_arrays(transform, operator, tau_s, state.divergence, state.theta,
                                      state.log_surface_pressure)
        if dataclasses.is_dataclass(state):
            return dataclasses.replace(state, divergence=d, theta=th, log_surface_pressure=lp)
        fields = list(state.fields())
        fields[1], fields[2], fields[3] = d, th, lp
        return state.with_fields(fields)
