// The trajectory deformation diagnostics of the semi-Lagrangian step
// (sht_lipschitz.cu): launcher shared with the C ABI in sht_semilag.cu.
#pragma once

#include "sht_common.cuh"

namespace sht {

// One advecting flow as the diagnostic reads it: vx, vy, vz (Cartesian wind,
// m/s) and the level rate (level indices per second), each
// [nlev][held rows][nlon], holding the grid's rows [held0, held0 + held).
template <typename T>
struct LipFlow {
  const T* f[4];
  int held0, held;
};

// Reduced results: maxima of the spectral, Frobenius, horizontal, vertical
// and balanced norms (per second), the minima of det(I + (dt/2) J) and
// det(I - (dt/2) J_ex), and the flat (level, arrival row, lon) index of
// each minimum (the first in that order among equal values).
struct LipResult {
  double maxima[5];
  double minima[2];
  long long argmin[2];
};

// Bytes of device scratch the launcher needs on an nlat x nlon grid
// (per-block partials, the reduced result, the row and column tables).
size_t lipschitz_scratch_bytes(int nlat, int nlon);

// The diagnostics of the arrival rows [a0, a1) of an nlat x nlon grid
// (lat_ext: the extended latitudes in T, row j at j + 2; the rows beyond a
// pole are read from the pole row half a turn round).  `ex` with
// ex.f[0] == nullptr: the arrival side reads `wind`.  Every neighbour row a
// derivative reads must be held (checked by the caller).  Synchronises
// `s` and fills `out`.
template <typename T>
void launch_lipschitz(int nlev, int nlat, int nlon, int a0, int a1, const T* lat_ext,
                      const LipFlow<T>& wind, const LipFlow<T>& ex, double dt_s,
                      double radius_m, double reference_length_m, void* scratch,
                      LipResult* out, cudaStream_t s);

}  // namespace sht
