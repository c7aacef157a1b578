"""Record the reference's semi-implicit maps and the vertical operator they use.

Run in the build container, where the reference source tree is mounted:

    python tests/golden/make_golden_semi.py <reference checkout>

For two cases (T7 with 6 levels, T21 with 40) it builds the reference's
``HybridCoordinate.pressure_blend`` stack and its ``VerticalModeSemiImplicit``
(default reference state; off-centring 0.5 and 0.55), runs ``solve_shifted``,
``apply``, ``half_apply`` and ``linear_tendencies`` on a seeded projected
state, records ``explicit_wave_speed_m_s`` and the modes ``describe`` reports,
and writes
``semi_<case>.npz`` with:

* the coordinate's half-level A and B and its hydrostatic geopotential
  response to a unit virtual temperature at each level (the one method of
  the coordinate the operator build calls; a GPU host without the reference
  answers it from this matrix);
* the operator's B, C, modes of M = -B C and of the thermodynamic block C B;
* inputs, outputs and the reported max divergence increments.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


class _State:
    """The ten fields the maps read and rebuild, with ``with_fields``."""

    def __init__(self, fields):
        (self.vorticity, self.divergence, self.theta, self.log_surface_pressure, self.qv,
         self.qc, self.qr, self.qi, self.qs, self.qg) = fields

    def with_fields(self, fields):
        return _State(tuple(fields))


def main(ref_root: str) -> None:
    root = Path(ref_root)
    os.environ.setdefault("ARWEN_GLOBAL_LEGENDRE_CACHE", "off")
    sys.path[:0] = [str(root / "src"), str(root / "tests")]
    from arwen_global.constants import DRY_AIR_GAS_CONSTANT
    from arwen_global.semi_implicit import VerticalModeSemiImplicit
    from arwen_global.spectral.transform import SphericalHarmonicTransform
    from arwen_global.vertical import HybridCoordinate

    for name, t, nlev, tau, dt in [("t7_l6", 7, 6, 1800.0, 1200.0),
                                   ("t21_l40", 21, 40, 300.0, 600.0)]:
        rng = np.random.default_rng(31 + nlev)
        transform = SphericalHarmonicTransform.create(t, precision="float64")
        vertical = HybridCoordinate.pressure_blend(nlev, 100.0)
        semi = VerticalModeSemiImplicit()
        semi55 = VerticalModeSemiImplicit(off_centring_weight=0.55, divergence_weight=0.9)
        op = semi.operator(vertical)
        ps_ref = semi.reference_surface_pressure_pa
        p_half = vertical.a_half_pa + vertical.b_half * ps_ref
        response = np.zeros((nlev, nlev))
        for j in range(nlev):
            unit = np.zeros((nlev, 1, 1))
            unit[j] = 1.0
            response[:, j] = vertical.hydrostatic_geopotential(
                unit, np.zeros((1, 1)), p_half[:, None, None],
                gas_constant=DRY_AIR_GAS_CONSTANT)[:, 0, 0]

        def field(shape, scale):
            return transform.project(scale * (rng.standard_normal(shape)
                                              + 1j * rng.standard_normal(shape)))

        shape = (nlev, t + 1, t + 1)
        qv = np.zeros(shape, dtype=np.complex128)
        state = _State((field(shape, 1e-5), field(shape, 1e-5), field(shape, 1.0),
                        field((t + 1, t + 1), 1e-3), qv, None, None, None, None, None))
        solved = semi.solve_shifted(state, transform, vertical, tau)
        applied, m_apply = semi.apply(state, transform, vertical, dt)
        applied55, m_apply55 = semi55.apply(state, transform, vertical, dt)
        half, m_half = semi.half_apply(state, transform, vertical, dt)
        half55, m_half55 = semi55.half_apply(state, transform, vertical, dt)
        lin = semi.linear_tendencies(state, transform, vertical)
        lin90 = semi55.linear_tendencies(state, transform, vertical)
        np.savez_compressed(
            HERE / f"semi_{name}.npz",
            truncation=t, nlev=nlev, tau_s=tau, dt_s=dt,
            radius_m=transform.grid.radius_m,
            reference_temperature_k=semi.reference_temperature_k,
            reference_surface_pressure_pa=ps_ref,
            a_half_pa=vertical.a_half_pa, b_half=vertical.b_half,
            geopotential_response=response,
            b_matrix=op.b_matrix, c_matrix=op.c_matrix,
            eigenvalues=op.eigenvalues, eigenvectors=op.eigenvectors,
            x_eigenvalues=op.x_eigenvalues, x_eigenvectors=op.x_eigenvectors,
            divergence=state.divergence, theta=state.theta,
            lnps=state.log_surface_pressure, vorticity=state.vorticity,
            solve_divergence=solved.divergence, solve_theta=solved.theta,
            solve_lnps=solved.log_surface_pressure,
            apply_divergence=applied.divergence, apply_theta=applied.theta,
            apply_lnps=applied.log_surface_pressure,
            apply_metric=m_apply["semi_implicit_max_divergence_increment_s1"],
            apply55_divergence=applied55.divergence, apply55_theta=applied55.theta,
            apply55_lnps=applied55.log_surface_pressure,
            apply55_metric=m_apply55["semi_implicit_max_divergence_increment_s1"],
            half_divergence=half.divergence, half_theta=half.theta,
            half_lnps=half.log_surface_pressure,
            half_metric=m_half["semi_implicit_max_divergence_increment_s1"],
            half55_divergence=half55.divergence, half55_theta=half55.theta,
            half55_lnps=half55.log_surface_pressure,
            half55_metric=m_half55["semi_implicit_max_divergence_increment_s1"],
            linear_divergence=lin.divergence, linear_theta=lin.theta,
            linear_lnps=lin.log_surface_pressure,
            linear90_divergence=lin90.divergence, linear90_theta=lin90.theta,
            linear90_lnps=lin90.log_surface_pressure,
            explicit_wave_speed_m_s=semi.explicit_wave_speed_m_s(vertical),
            explicit90_wave_speed_m_s=semi55.explicit_wave_speed_m_s(vertical),
            phase_speeds_m_s=np.asarray(semi.describe(vertical)["phase_speeds_m_s"]),
            equivalent_depths_m=np.asarray(semi.describe(vertical)["equivalent_depths_m"]),
        )
        print("wrote semi", name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path to the reference checkout>")
    main(sys.argv[1])
