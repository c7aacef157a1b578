"""Helpers shared by the semi-implicit tests (no test functions here)."""
from __future__ import annotations

import numpy as np


class RecordedCoordinate:
    """A stand-in for the reference's ``HybridCoordinate`` on a host without
    the reference: its half-level A/B and its hydrostatic integration,
    answered from the geopotential response to a unit virtual temperature at
    each level that the fixture script recorded from the coordinate itself
    (the integration is linear in Tv at fixed pressure)."""

    def __init__(self, g):
        self.a_half_pa = np.asarray(g["a_half_pa"], dtype=np.float64)
        self.b_half = np.asarray(g["b_half"], dtype=np.float64)
        self.nlev = int(g["nlev"])
        self._response = np.asarray(g["geopotential_response"], dtype=np.float64)

    def hydrostatic_geopotential(self, virtual_temperature, surface_geopotential, p_half, *,
                                 gas_constant=287.0):
        t = np.asarray(virtual_temperature, dtype=np.float64)
        phi = np.tensordot(self._response, t, axes=([1], [0]))
        return phi + np.asarray(surface_geopotential)[None]


class State:
    """The ten fields of the reference's state that the maps read and rebuild."""

    def __init__(self, fields):
        (self.vorticity, self.divergence, self.theta, self.log_surface_pressure, self.qv,
         self.qc, self.qr, self.qi, self.qs, self.qg) = fields

    def with_fields(self, fields):
        return State(tuple(fields))

    @classmethod
    def from_golden(cls, g):
        return cls((g["vorticity"], g["divergence"], g["theta"], g["lnps"], None, None, None,
                    None, None, None))
