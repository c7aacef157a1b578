// Semi-Lagrangian interpolation at departure points on the Gaussian grid:
// the tricubic (4 x 4 x 4) and quintic-horizontal (6 x 6 x 4) gathers with
// the quasi-monotone limiter and its clip deficit, and the trilinear gather
// inside the limiter's cell (the reference's semilag/kernels.cu entry
// families sl_gather_*, sl_gather5_*, sl_linear_*; their numpy
// specification is semilag/interpolate.py:505-725, the tables
// semilag/tables.py:51-236).
//
// Geometry of the stencil (the reference's conventions, which a drop-in
// must keep):
//   * zonal: uniform nodes lon[i] = 2 pi i / nlon, periodic; the departure
//     point is a continuous zonal index; equispaced Lagrange weights;
//   * meridional: the Gauss nodes extended by NH/2 reflected rows beyond
//     each pole (a row past a pole is the ring on the other
//     side read half a turn round), Lagrange weights on the true node
//     latitudes from reciprocal denominators tabulated per stencil start;
//   * vertical: four-point cubic in the continuous level index, the index
//     clamped to the boundary interfaces [-1/2, nlev - 1/2], the stencil
//     start to [0, nlev - 4];
//   * every weight set normalised by its sum (exact identity at a node);
//   * taps summed as differences from the stencil node nearest the point,
//     the centre added back once;
//   * unlimited fields: the half layer outside the outermost full level is
//     held between that level's value and the linear reconstruction at the
//     interface; limited fields: clipped to the [min, max] of the 2 x 2 x 2
//     cell around the point, the deficit being raw - kept.
//
// B200 layout: one thread per arrival point, consecutive threads along a
// latitude row (the departure points of a warp are neighbours, so its tap
// loads share cache lines), rows taken with all their levels together (the
// four arrival levels whose stencils read one source level plane run at the
// same time, so the plane comes from DRAM about once); the geometry tables
// (a few tens of KB) are read through the read-only path; in-plane offsets
// are 32-bit; the F fields of one call share the index and weight
// computation, two fields per pass on the four-point stencil.  The gather is bound by
// its tap loads (64 or 144 per point per field, nearly all L1/L2 hits) and
// by HBM for the coordinates, sources and outputs.
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "sht_common.cuh"
#include "sht_lipschitz.h"

struct SlWidth {
  int ghost = 0;                // reflected rows beyond each pole
  int rows = 0;                 // extended rows: nlat + 2 ghost
  int bins = 0;                 // bracket lookup bins
  double lut_scale = 0.0;       // bins per radian
  std::vector<double> lat_ext;  // [rows]
  std::vector<double> mrden;    // [(nlat + 1) x NH]
  std::vector<int32_t> mlut, rowoff, rowshift;
  void* d_lat_ext = nullptr;    // element type of the tables
  void* d_mrden = nullptr;
  int32_t* d_mlut = nullptr;
  int32_t* d_rowoff = nullptr;
  int32_t* d_rowshift = nullptr;
};

struct sht_sl_tables {
  int nlat = 0, nlon = 0, prec = 0, device = 0;
  SlWidth w4, w6;  // w6 empty when nlat < 6
  void* d_lip = nullptr;  // scratch of the deformation diagnostic, made on first use
};

// One latitude band of a semi-Lagrangian step: arrival rows [a0, a1) read
// from fields that hold rows [s0, s1) (the band and its halo).  The row
// offsets of both stencil widths are rebased to the held rows (-1 for a
// row outside them); the weights and brackets stay the whole grid's, so a
// band computes the whole-grid values bit for bit.
struct sht_sl_window {
  const sht_sl_tables* tables = nullptr;
  int s0 = 0, s1 = 0, a0 = 0, a1 = 0;
  int32_t* d_rowoff4 = nullptr;
  int32_t* d_rowoff6 = nullptr;
  int* d_esc = nullptr;  // escape flag
};

namespace sht {
namespace {

template <class F>
int guarded(F&& f) {
  try {
    clear_error();
    f();
    return SHT_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    set_error(e.what());
    return SHT_ERR_STATE;
  }
}

constexpr double kHalfPi = 1.57079632679489661923;
// Departure-point solvers (the reference's TRAJECTORY_SOLVERS, in order).
constexpr int kSolverFixedPoint = 0;
constexpr int kSolverNewton = 1;
constexpr int kSolverNewtonLs = 2;

// ------------------------------------------------------------- weights

// Lagrange weights on the equispaced nodes 0 .. NH-1 at t, normalised.
template <typename T, int NH>
__device__ __forceinline__ void equispaced_weights(T t, T (&w)[NH]) {
  if constexpr (NH == 4) {
    const T d0 = t, d1 = t - T(1), d2 = t - T(2), d3 = t - T(3);
    w[0] = -d1 * d2 * d3 * T(1.0 / 6.0);
    w[1] = d0 * d2 * d3 * T(0.5);
    w[2] = -d0 * d1 * d3 * T(0.5);
    w[3] = d0 * d1 * d2 * T(1.0 / 6.0);
  } else {
    T d[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) d[q] = t - T(q);
    // 1 / prod_{q != m} (m - q): -1/120, 1/24, -1/12, 1/12, -1/24, 1/120
    const T c[6] = {T(-1.0 / 120.0), T(1.0 / 24.0), T(-1.0 / 12.0),
                    T(1.0 / 12.0),   T(-1.0 / 24.0), T(1.0 / 120.0)};
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      T prod = T(1);
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (q != m) prod *= d[q];
      w[m] = prod * c[m];
    }
  }
  T sum = w[0];
#pragma unroll
  for (int q = 1; q < NH; ++q) sum += w[q];
  const T inv = T(1) / sum;
#pragma unroll
  for (int q = 0; q < NH; ++q) w[q] *= inv;
}

// The extended row m0 with lat_ext[m0] <= p < lat_ext[m0 + 1], held in
// [G, nj + G] (G = 1 for the four-row stencil m0-1 .. m0+2, 2 for the
// six-row stencil m0-2 .. m0+3) so that the stencil stays in the table: a
// lookup bin, then exact steps (zero or one for Gauss nodes).
template <typename T>
__device__ __forceinline__ int bracket(T p, const T* __restrict__ lat_ext,
                                       const int32_t* __restrict__ mlut, int nb, int nj, int G,
                                       T lut_scale) {
  int b = (int)((p + T(kHalfPi)) * lut_scale);
  b = min(max(b, 0), nb - 1);
  int m0 = __ldg(mlut + b);
  while (m0 > G && p < __ldg(lat_ext + m0)) --m0;
  while (m0 < nj + G && p >= __ldg(lat_ext + m0 + 1)) ++m0;
  return m0;
}

// Memory index (k, j, i) of the t-th point in (j, k, i) order.
// (Below 2^31 points, which the host checks: 32-bit divisions.)
__device__ __forceinline__ int64_t point_index(int64_t t, int nk, int nj, int ni) {
  const unsigned u = (unsigned)t;
  const unsigned r = u / (unsigned)ni;
  const unsigned i = u - r * (unsigned)ni;
  const unsigned j = r / (unsigned)nk;
  const unsigned k = r - j * (unsigned)nk;
  return ((int64_t)k * nj + j) * ni + i;
}

template <typename T>
struct SlArgs {
  const T* src;    // [F][nk][nj][ni]
  const T* xi;     // [nk][nj][ni] continuous zonal index
  const T* phi;    // latitude, radians
  const T* lev;    // continuous full-level index
  const T* lat_ext;
  const T* mrden;
  const int32_t* mlut;
  const int32_t* rowoff;
  const int32_t* rowshift;
  T* out;          // [F][nk][nja][ni]
  T* cut;          // clip deficit (or null)
  int F, nk, nj, ni, nb;
  T lut_scale;
  // Latitude-band form: the sources hold njs rows (the band and its halo),
  // the coordinates and outputs the band's nja rows; rowoff then maps an
  // extended row to its offset inside the held rows, or to -1 for a row
  // the band does not hold (a read of it sets *esc and reads row 0).  On
  // the whole grid njs = nja = nj and esc is null.
  int njs, nja;
  int* esc;
};

// The in-plane offset of extended row r: an offset of -1 (a row outside a
// band's held rows) raises the escape flag and reads the first held row,
// so the access stays in bounds while the caller refuses the result.
__device__ __forceinline__ int held_row(const int32_t* __restrict__ rowoff, int r, int* esc) {
  int ro = __ldg(rowoff + r);
  if (ro < 0) {
    if (esc) atomicOr(esc, 1);
    ro = 0;
  }
  return ro;
}

// --------------------------------------------------------------- gather
template <typename T, int NH, bool QM, bool DEF>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 && NH == 4) ? 3 : 2) sl_gather_kernel(const SlArgs<T> a) {
  constexpr int G = NH / 2 - 1;  // zonal lead and meridional start offset
  constexpr int MID = NH / 2 - 1;
  const int plane = a.njs * a.ni;              // a held source level
  const int64_t n = (int64_t)a.nk * a.nja * a.ni;  // arrival points
  // Threads walk the points row by row with the levels of a row together:
  // a source level plane is read by the stencils of four arrival levels,
  // which then run at the same time and find it in L2 (level-major order
  // brought every plane in from DRAM about four times).
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t gid = point_index(t, a.nk, a.nja, a.ni);

  const T p = min(max(a.phi[gid], T(-kHalfPi)), T(kHalfPi));
  const T xk = min(max(a.lev[gid], T(-0.5)), T(a.nk) - T(0.5));
  const bool below = xk < T(0);
  const bool outside = below || xk > T(a.nk - 1);
  const int c_edge = below ? 0 : 3, c_next = below ? 1 : 2;
  const T xi = a.xi[gid];

  // zonal: periodic, never clamped
  const T fi = floor(xi);
  const int i0 = (int)fi - G;
  T wx[NH];
  equispaced_weights<T, NH>(xi - T(i0), wx);
  int col[NH], colh[NH];
  col[0] = i0 % a.ni;
  if (col[0] < 0) col[0] += a.ni;
#pragma unroll
  for (int q = 1; q < NH; ++q) col[q] = col[q - 1] + 1 == a.ni ? 0 : col[q - 1] + 1;
  const int half = a.ni >> 1;
#pragma unroll
  for (int q = 0; q < NH; ++q) colh[q] = col[q] >= a.ni - half ? col[q] + half - a.ni : col[q] + half;

  // meridional: true nodes, the poles by reflection
  const int sst = bracket<T>(p, a.lat_ext, a.mlut, a.nb, a.nj, G, a.lut_scale) - G;
  T d[NH], wy[NH];
#pragma unroll
  for (int m = 0; m < NH; ++m) d[m] = p - __ldg(a.lat_ext + sst + m);
  {
    T sum = T(0);
#pragma unroll
    for (int m = 0; m < NH; ++m) {
      T prod = T(1);
      bool first = true;
#pragma unroll
      for (int q = 0; q < NH; ++q) {
        if (q == m) continue;
        prod = first ? d[q] : prod * d[q];
        first = false;
      }
      wy[m] = prod * __ldg(a.mrden + NH * sst + m);
      sum = m == 0 ? wy[0] : sum + wy[m];
    }
    const T inv = T(1) / sum;
#pragma unroll
    for (int m = 0; m < NH; ++m) wy[m] *= inv;
  }

  // vertical: uniform in the level index, start clamped to the data
  const int kb = min(max((int)floor(xk), 0), a.nk - 2);
  const int k0 = min(max(kb - 1, 0), a.nk - 4);
  const int kbox = kb - k0;
  T wz[4];
  equispaced_weights<T, 4>(xk - T(k0), wz);

  int adr[NH][NH];  // in-plane offsets of the stencil's taps
#pragma unroll
  for (int m = 0; m < NH; ++m) {
    const int ro = held_row(a.rowoff, sst + m, a.esc);
    const bool sh = __ldg(a.rowshift + sst + m) != 0;
#pragma unroll
    for (int q = 0; q < NH; ++q) adr[m][q] = ro + (sh ? colh[q] : col[q]);
  }
  // the node nearest the point in each direction
  const int cx = (xi - fi >= T(0.5)) ? MID + 1 : MID;
  const int cy = (d[MID] >= __ldg(a.lat_ext + sst + MID + 1) - p) ? MID + 1 : MID;
  const int kn = min(max((int)floor(xk + T(0.5)), 0), a.nk - 1);
  int centre = adr[MID][MID];
#pragma unroll
  for (int m = MID; m <= MID + 1; ++m)
#pragma unroll
    for (int q = MID; q <= MID + 1; ++q)
      if (m == cy && q == cx) centre = adr[m][q];

  const int64_t fstride = n;                          // output field stride
  const int64_t sstride = (int64_t)a.nk * plane;       // source field stride
  const int64_t cofs = (int64_t)kn * plane + centre;
  // NB fields per pass share every address; their taps are in flight
  // together, two levels at a time (a fully unrolled level loop holds every
  // level's loads and weights at once, 180+ registers; one level at a time
  // measured 4-14 % slower).
  auto fields = [&](auto nb_tag, int f0) {
    constexpr int NB = decltype(nb_tag)::value;
    const T* s[NB];
    T base[NB], acc[NB], lo[NB], hi[NB], f_edge[NB], f_next[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      s[b] = a.src + (f0 + b) * sstride;
      base[b] = __ldg(s[b] + cofs);
      acc[b] = lo[b] = hi[b] = f_edge[b] = f_next[b] = T(0);
    }
    bool boxed = false;
#pragma unroll 2
    for (int c = 0; c < 4; ++c) {
      const int64_t lofs = (int64_t)(k0 + c) * plane;
      const T wzc = c == 0 ? wz[0] : (c == 1 ? wz[1] : (c == 2 ? wz[2] : wz[3]));
      const bool inbox = QM && (c == kbox || c == kbox + 1);
      T rowsum[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) rowsum[b] = T(0);
#pragma unroll
      for (int m = 0; m < NH; ++m) {
        T v[NB][NH];
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
          for (int q = 0; q < NH; ++q) v[b][q] = __ldg(s[b] + lofs + adr[m][q]);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          if (inbox && (m == MID || m == MID + 1)) {
            const T vmin = min(v[b][MID], v[b][MID + 1]), vmax = max(v[b][MID], v[b][MID + 1]);
            lo[b] = boxed ? min(lo[b], vmin) : vmin;
            hi[b] = boxed ? max(hi[b], vmax) : vmax;
          }
          T colsum = wx[0] * (v[b][0] - base[b]);
#pragma unroll
          for (int q = 1; q < NH; ++q) colsum += wx[q] * (v[b][q] - base[b]);
          rowsum[b] += wy[m] * colsum;
        }
        if (inbox && (m == MID || m == MID + 1)) boxed = true;
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        acc[b] += wzc * rowsum[b];
        if (c == c_edge) f_edge[b] = rowsum[b];
        if (c == c_next) f_next[b] = rowsum[b];
      }
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      T r = acc[b];
      if (!QM && outside) {
        const T f_face = f_edge[b] + T(0.5) * (f_edge[b] - f_next[b]);
        r = min(max(r, min(f_edge[b], f_face)), max(f_edge[b], f_face));
      }
      r += base[b];
      const T kept = QM ? min(max(r, lo[b]), hi[b]) : r;
      a.out[(f0 + b) * fstride + gid] = kept;
      if (DEF) a.cut[(f0 + b) * fstride + gid] = r - kept;
    }
  };
  // Two fields per pass on the four-point stencil; the six-point one
  // takes one (two would hold 190+ registers).
  constexpr int NB = NH == 4 ? 2 : 1;
  int f = 0;
  for (; f + NB <= a.F; f += NB) fields(std::integral_constant<int, NB>{}, f);
  if (f < a.F) fields(std::integral_constant<int, 1>{}, f);
}

// ------------------------------------------------------------ trilinear
// Inside the limiter's cell: columns floor(xi), +1; extended rows m0, m0+1
// of the cubic bracket; levels kb, kb+1 with the index held in [0, nk-1].
template <typename T>
__global__ void __launch_bounds__(256) sl_linear_kernel(const SlArgs<T> a) {
  const int plane = a.nj * a.ni;
  const int64_t n = (int64_t)a.nk * plane;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t gid = point_index(t, a.nk, a.nj, a.ni);  // rows with their levels together
  const T p = min(max(a.phi[gid], T(-kHalfPi)), T(kHalfPi));
  const T xk = min(max(a.lev[gid], T(0)), T(a.nk - 1));
  const T xi = a.xi[gid];
  const T fi = floor(xi);
  const T ax = xi - fi;
  int c0 = ((int)fi) % a.ni;
  if (c0 < 0) c0 += a.ni;
  const int c1 = c0 + 1 == a.ni ? 0 : c0 + 1;
  const int half = a.ni >> 1;
  const int h0 = c0 >= a.ni - half ? c0 + half - a.ni : c0 + half;
  const int h1 = c1 >= a.ni - half ? c1 + half - a.ni : c1 + half;
  const int m0 = bracket<T>(p, a.lat_ext, a.mlut, a.nb, a.nj, 1, a.lut_scale);
  const T la = __ldg(a.lat_ext + m0), lb = __ldg(a.lat_ext + m0 + 1);
  const T ay = min(max((p - la) / (lb - la), T(0)), T(1));
  const int r0 = __ldg(a.rowoff + m0), r1 = __ldg(a.rowoff + m0 + 1);
  const bool s0 = __ldg(a.rowshift + m0) != 0, s1 = __ldg(a.rowshift + m0 + 1) != 0;
  const int i00 = r0 + (s0 ? h0 : c0), i01 = r0 + (s0 ? h1 : c1);
  const int i10 = r1 + (s1 ? h0 : c0), i11 = r1 + (s1 ? h1 : c1);
  const int kb = min(max((int)floor(xk), 0), a.nk - 2);
  const T az = xk - T(kb);
  const T bx = T(1) - ax, by = T(1) - ay, bz = T(1) - az;
  for (int f = 0; f < a.F; ++f) {
    const T* s0p = a.src + f * n + (int64_t)kb * plane;
    const T* s1p = s0p + plane;
    const T t0 = by * (bx * __ldg(s0p + i00) + ax * __ldg(s0p + i01)) +
                 ay * (bx * __ldg(s0p + i10) + ax * __ldg(s0p + i11));
    const T t1 = by * (bx * __ldg(s1p + i00) + ax * __ldg(s1p + i01)) +
                 ay * (bx * __ldg(s1p + i10) + ax * __ldg(s1p + i11));
    a.out[f * n + gid] = bz * t0 + az * t1;
  }
}

// ------------------------------------------------------ departure search
// The fixed-point departure-point search of the reference
// (semilag/trajectory.py:553-618, kernels.cu sl_departure_*), all
// iterations in one launch: with a the arrival point's unit vector, V the
// Cartesian wind (m/s) and s the level rate (levels/s) at full levels,
//   first guess  q = normalize(a - dt V(a) / r),  k_q = k - dt s(a);
//   iteration    q' = normalize(a - dt/2 (V_ex(a) + V(q)) / r),
//                k_q' = k - dt/2 (s_ex(a) + s(q, k_q)),
// V(q), s(q) read trilinearly in the cubic gather's cell, levels clamped to
// the boundary interfaces [-1/2, nlev - 1/2].  Outputs the departure
// coordinates (continuous zonal index, latitude, level) and the last
// iteration's move (metres along the great circle, levels).
template <typename T>
struct SlDepArgs {
  const T *vx, *vy, *vz, *sv;      // advecting wind [nk][nj][ni]
  const T *vxe, *vye, *vze, *sve;  // extrapolated wind at the arrival points
  const T* lat_ext;
  const int32_t *mlut, *rowoff, *rowshift;
  T *xi, *phi, *lev, *move_m, *move_k;
  int iters, nk, nj, ni, nb;
  double dlam;  // 2 pi / nlon (the arrival longitudes are formed in double)
  T dt, radius, inv_dlam, lut_scale;
  // Latitude-band form: the advecting wind holds njs rows starting `lead`
  // rows above the first arrival row, grid row ja0; the extrapolated wind
  // and the outputs hold the nja arrival rows.  Whole grid: njs = nja = nj,
  // ja0 = lead = 0, esc null.
  int njs, nja, ja0, lead;
  int* esc;
};

template <typename T>
__device__ __forceinline__ void trilinear4(const SlDepArgs<T>& a, T lam, T phid, T xkd,
                                           T (&w)[4]) {
  const T p = min(max(phid, T(-kHalfPi)), T(kHalfPi));
  const T xk = min(max(xkd, T(0)), T(a.nk - 1));
  const T x = lam * a.inv_dlam;
  const T fi = floor(x);
  const T ax = x - fi;
  int c0 = ((int)fi) % a.ni;
  if (c0 < 0) c0 += a.ni;
  const int c1 = c0 + 1 == a.ni ? 0 : c0 + 1;
  const int half = a.ni >> 1;
  const int h0 = c0 >= a.ni - half ? c0 + half - a.ni : c0 + half;
  const int h1 = c1 >= a.ni - half ? c1 + half - a.ni : c1 + half;
  const int m0 = bracket<T>(p, a.lat_ext, a.mlut, a.nb, a.nj, 1, a.lut_scale);
  const T la = __ldg(a.lat_ext + m0), lb = __ldg(a.lat_ext + m0 + 1);
  const T ay = (p - la) / (lb - la);
  const int r0 = held_row(a.rowoff, m0, a.esc), r1 = held_row(a.rowoff, m0 + 1, a.esc);
  const bool s0 = __ldg(a.rowshift + m0) != 0, s1 = __ldg(a.rowshift + m0 + 1) != 0;
  const int i00 = r0 + (s0 ? h0 : c0), i01 = r0 + (s0 ? h1 : c1);
  const int i10 = r1 + (s1 ? h0 : c0), i11 = r1 + (s1 ? h1 : c1);
  const int k0 = min(max((int)floor(xk), 0), a.nk - 2);
  const T az = xk - T(k0);
  const int64_t plane = (int64_t)a.njs * a.ni;
  const int64_t o0 = (int64_t)k0 * plane, o1 = o0 + plane;
  const T bx = T(1) - ax, by = T(1) - ay, bz = T(1) - az;
  const T* f[4] = {a.vx, a.vy, a.vz, a.sv};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const T* s0p = f[q] + o0;
    const T* s1p = f[q] + o1;
    const T t0 = by * (bx * __ldg(s0p + i00) + ax * __ldg(s0p + i01)) +
                 ay * (bx * __ldg(s0p + i10) + ax * __ldg(s0p + i11));
    const T t1 = by * (bx * __ldg(s1p + i00) + ax * __ldg(s1p + i01)) +
                 ay * (bx * __ldg(s1p + i10) + ax * __ldg(s1p + i11));
    w[q] = bz * t0 + az * t1;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) sl_departure_kernel(const SlDepArgs<T> a) {
  const int64_t n = (int64_t)a.nk * a.nja * a.ni;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t gid = point_index(t, a.nk, a.nja, a.ni);  // rows with their levels together
  const int plane = a.nja * a.ni;
  const int k = (int)(gid / plane);
  const int rem = (int)(gid - (int64_t)k * plane);
  const int j = rem / a.ni, i = rem - j * a.ni;
  // the arrival point in the advecting wind's held rows
  const int64_t here = ((int64_t)k * a.njs + (j + a.lead)) * a.ni + i;
  // the arrival point: table latitude and i * dlam (formed in double, as
  // the host computes the grid's longitudes), both in T
  const T lat = __ldg(a.lat_ext + a.ja0 + j + 2);
  const T lon = T((double)i * a.dlam);
  const T sph = sin(lat), cph = cos(lat), sla = sin(lon), cla = cos(lon);
  const T ax = cph * cla, ay = cph * sla, az = sph;
  const T inv_r = T(1) / a.radius;
  const T dt = a.dt, hdt = T(0.5) * a.dt;
  T qx = ax - dt * a.vx[here] * inv_r;
  T qy = ay - dt * a.vy[here] * inv_r;
  T qz = az - dt * a.vz[here] * inv_r;
  T nrm = sqrt(qx * qx + qy * qy + qz * qz);
  qx /= nrm;
  qy /= nrm;
  qz /= nrm;
  const T klo = T(-0.5), khi = T(a.nk) - T(0.5);
  T qk = min(max(T(k) - dt * a.sv[here], klo), khi);
  const T ex = a.vxe[gid], ey = a.vye[gid], ez = a.vze[gid], es = a.sve[gid];
  T last_m = T(0), last_k = T(0);
  for (int it = 0; it < a.iters; ++it) {
    const T lam = atan2(qy, qx);
    const T phid = atan2(qz, sqrt(qx * qx + qy * qy));
    T w[4];
    trilinear4<T>(a, lam, phid, qk, w);
    T px = ax - hdt * (ex + w[0]) * inv_r;
    T py = ay - hdt * (ey + w[1]) * inv_r;
    T pz = az - hdt * (ez + w[2]) * inv_r;
    nrm = sqrt(px * px + py * py + pz * pz);
    px /= nrm;
    py /= nrm;
    pz /= nrm;
    const T pk = min(max(T(k) - hdt * (es + w[3]), klo), khi);
    const T cx = px - qx, cy = py - qy, cz = pz - qz;
    const T chord = sqrt(cx * cx + cy * cy + cz * cz);
    last_m = a.radius * T(2) * asin(min(max(T(0.5) * chord, T(0)), T(1)));
    last_k = fabs(pk - qk);
    qx = px;
    qy = py;
    qz = pz;
    qk = pk;
  }
  a.xi[gid] = atan2(qy, qx) * a.inv_dlam;
  a.phi[gid] = atan2(qz, sqrt(qx * qx + qy * qy));
  a.lev[gid] = qk;
  a.move_m[gid] = last_m;
  a.move_k[gid] = last_k;
}

// ------------------------------------------------ Newton departure search
// The same departure equation solved by Newton's method (the reference's
// opt-in "newton" solver, semilag/trajectory.py TRAJECTORY_SOLVERS): with
// the fixed-point map G(q, k) above, find q, k with G(q, k) = (q, k).  At
// the current point the residual r = G - (q, k) is taken in the local
// east / north / level frame, the Jacobian M of G in that frame comes from
// the trilinear interpolant's own derivatives (dV/d(east) = dV/dlambda /
// cos phi, dV/d(north) = dV/dphi, dV/dk; the normalisation's projection is
// dropped, exact at the solution), and (I - M) d = r is solved by Cramer's
// rule.  A step is taken only where det(I - M) > 0.05 and cos phi > 1e-6
// and it is at most five times the plain step; otherwise, and where the
// residual did not shrink, the plain fixed-point step d = r is taken.  Both
// solvers share one fixed point.
template <typename T>
__device__ __forceinline__ void trilinear4_grad(const SlDepArgs<T>& a, T lam, T phid, T xkd,
                                                T (&w)[4], T (&dl)[4], T (&dp)[4], T (&dk)[4]) {
  const T p = min(max(phid, T(-kHalfPi)), T(kHalfPi));
  const bool kclamp = xkd <= T(0) || xkd >= T(a.nk - 1);
  const T xk = min(max(xkd, T(0)), T(a.nk - 1));
  const T x = lam * a.inv_dlam;
  const T fi = floor(x);
  const T ax = x - fi;
  int c0 = ((int)fi) % a.ni;
  if (c0 < 0) c0 += a.ni;
  const int c1 = c0 + 1 == a.ni ? 0 : c0 + 1;
  const int half = a.ni >> 1;
  const int h0 = c0 >= a.ni - half ? c0 + half - a.ni : c0 + half;
  const int h1 = c1 >= a.ni - half ? c1 + half - a.ni : c1 + half;
  const int m0 = bracket<T>(p, a.lat_ext, a.mlut, a.nb, a.nj, 1, a.lut_scale);
  const T la = __ldg(a.lat_ext + m0), lb = __ldg(a.lat_ext + m0 + 1);
  const T inv_dphi = T(1) / (lb - la);
  const T ay = (p - la) * inv_dphi;
  const int r0 = held_row(a.rowoff, m0, a.esc), r1 = held_row(a.rowoff, m0 + 1, a.esc);
  const bool s0 = __ldg(a.rowshift + m0) != 0, s1 = __ldg(a.rowshift + m0 + 1) != 0;
  const int i00 = r0 + (s0 ? h0 : c0), i01 = r0 + (s0 ? h1 : c1);
  const int i10 = r1 + (s1 ? h0 : c0), i11 = r1 + (s1 ? h1 : c1);
  const int k0 = min(max((int)floor(xk), 0), a.nk - 2);
  const T az = xk - T(k0);
  const int64_t plane = (int64_t)a.njs * a.ni;
  const int64_t o0 = (int64_t)k0 * plane, o1 = o0 + plane;
  const T bx = T(1) - ax, by = T(1) - ay, bz = T(1) - az;
  const T* f[4] = {a.vx, a.vy, a.vz, a.sv};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const T* u = f[q] + o0;
    const T* v = f[q] + o1;
    const T u00 = __ldg(u + i00), u01 = __ldg(u + i01), u10 = __ldg(u + i10), u11 = __ldg(u + i11);
    const T v00 = __ldg(v + i00), v01 = __ldg(v + i01), v10 = __ldg(v + i10), v11 = __ldg(v + i11);
    const T t0 = by * (bx * u00 + ax * u01) + ay * (bx * u10 + ax * u11);
    const T t1 = by * (bx * v00 + ax * v01) + ay * (bx * v10 + ax * v11);
    w[q] = bz * t0 + az * t1;
    const T gx0 = by * (u01 - u00) + ay * (u11 - u10), gx1 = by * (v01 - v00) + ay * (v11 - v10);
    const T gy0 = (bx * u10 + ax * u11) - (bx * u00 + ax * u01);
    const T gy1 = (bx * v10 + ax * v11) - (bx * v00 + ax * v01);
    dl[q] = (bz * gx0 + az * gx1) * a.inv_dlam;
    dp[q] = (bz * gy0 + az * gy1) * inv_dphi;
    dk[q] = kclamp ? T(0) : t1 - t0;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) sl_departure_newton_kernel(const SlDepArgs<T> a) {
  const int64_t n = (int64_t)a.nk * a.nja * a.ni;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t gid = point_index(t, a.nk, a.nja, a.ni);
  const int plane = a.nja * a.ni;
  const int k = (int)(gid / plane);
  const int rem = (int)(gid - (int64_t)k * plane);
  const int j = rem / a.ni, i = rem - j * a.ni;
  const int64_t here = ((int64_t)k * a.njs + (j + a.lead)) * a.ni + i;
  const T lat = __ldg(a.lat_ext + a.ja0 + j + 2);
  const T lon = T((double)i * a.dlam);
  const T ax = cos(lat) * cos(lon), ay = cos(lat) * sin(lon), az = sin(lat);
  const T inv_r = T(1) / a.radius;
  const T dt = a.dt, hdt = T(0.5) * a.dt, c = hdt * inv_r;
  // the fixed-point search's first guess
  T qx = ax - dt * a.vx[here] * inv_r, qy = ay - dt * a.vy[here] * inv_r,
    qz = az - dt * a.vz[here] * inv_r;
  T nrm = sqrt(qx * qx + qy * qy + qz * qz);
  qx /= nrm; qy /= nrm; qz /= nrm;
  const T klo = T(-0.5), khi = T(a.nk) - T(0.5);
  T qk = min(max(T(k) - dt * a.sv[here], klo), khi);
  const T ex = a.vxe[gid], ey = a.vye[gid], ez = a.vze[gid], es = a.sve[gid];
  const T cells = T(a.nj) / T(2 * kHalfPi);  // meridional grid lengths per radian
  T last_m = T(0), last_k = T(0), res_prev = T(-1);
  for (int it = 0; it < a.iters; ++it) {
    const T lam = atan2(qy, qx);
    const T rho = sqrt(qx * qx + qy * qy);
    const T phid = atan2(qz, rho);
    T w[4], dl[4], dp[4], dk[4];
    trilinear4_grad<T>(a, lam, phid, qk, w, dl, dp, dk);
    const T ux = ax - c * (ex + w[0]), uy = ay - c * (ey + w[1]), uz = az - c * (ez + w[2]);
    const T un = sqrt(ux * ux + uy * uy + uz * uz);
    const T px = ux / un, py = uy / un, pz = uz / un;
    const T pk = min(max(T(k) - hdt * (es + w[3]), klo), khi);
    const bool kheld = pk <= klo || pk >= khi;
    // local frame at q: east e, north nv
    const T cl = rho > T(0) ? qx / rho : T(1), sl = rho > T(0) ? qy / rho : T(0);
    const T cp = rho, sp = qz;
    const T e0 = -sl, e1 = cl;
    const T n0 = -sp * cl, n1 = -sp * sl, n2 = cp;
    const T dx = px - qx, dy = py - qy, dz = pz - qz;
    const T re = e0 * dx + e1 * dy, rn = n0 * dx + n1 * dy + n2 * dz, rk = pk - qk;
    T de = re, dn = rn, dkk = rk;
    const T res = sqrt((re * re + rn * rn) * cells * cells + rk * rk);
    const bool shrinking = res_prev < T(0) || res <= T(0.9) * res_prev;
    res_prev = res;
    if (shrinking && cp > T(1e-6)) {
      const T g = -c / un;
      const T icp = T(1) / cp;
      // M[r][col]: rows east, north, level; columns d(east), d(north), d(level)
      const T m00 = g * (e0 * dl[0] + e1 * dl[1]) * icp;
      const T m01 = g * (e0 * dp[0] + e1 * dp[1]);
      const T m02 = g * (e0 * dk[0] + e1 * dk[1]);
      const T m10 = g * (n0 * dl[0] + n1 * dl[1] + n2 * dl[2]) * icp;
      const T m11 = g * (n0 * dp[0] + n1 * dp[1] + n2 * dp[2]);
      const T m12 = g * (n0 * dk[0] + n1 * dk[1] + n2 * dk[2]);
      const T m20 = kheld ? T(0) : -hdt * dl[3] * icp;
      const T m21 = kheld ? T(0) : -hdt * dp[3];
      const T m22 = kheld ? T(0) : -hdt * dk[3];
      const T a00 = T(1) - m00, a01 = -m01, a02 = -m02;
      const T a10 = -m10, a11 = T(1) - m11, a12 = -m12;
      const T a20 = -m20, a21 = -m21, a22 = T(1) - m22;
      const T det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) +
                    a02 * (a10 * a21 - a11 * a20);
      if (isfinite(det) && det > T(0.05)) {
        const T id = T(1) / det;
        const T s0 = (re * (a11 * a22 - a12 * a21) - a01 * (rn * a22 - a12 * rk) +
                      a02 * (rn * a21 - a11 * rk)) * id;
        const T s1 = (a00 * (rn * a22 - a12 * rk) - re * (a10 * a22 - a12 * a20) +
                      a02 * (a10 * rk - rn * a20)) * id;
        const T s2 = (a00 * (a11 * rk - rn * a21) - a01 * (a10 * rk - rn * a20) +
                      re * (a10 * a21 - a11 * a20)) * id;
        const T step = sqrt((s0 * s0 + s1 * s1) * cells * cells + s2 * s2);
        if (isfinite(step) && step <= T(5) * res + T(1e-30)) {
          de = s0;
          dn = s1;
          dkk = s2;
        }
      }
    }
    T nx = qx + de * e0 + dn * n0, ny = qy + de * e1 + dn * n1, nz = qz + dn * n2;
    nrm = sqrt(nx * nx + ny * ny + nz * nz);
    nx /= nrm; ny /= nrm; nz /= nrm;
    const T nk = min(max(qk + dkk, klo), khi);
    const T cx = nx - qx, cy = ny - qy, cz = nz - qz;
    const T chord = sqrt(cx * cx + cy * cy + cz * cz);
    last_m = a.radius * T(2) * asin(min(max(T(0.5) * chord, T(0)), T(1)));
    last_k = fabs(nk - qk);
    qx = nx; qy = ny; qz = nz; qk = nk;
  }
  a.xi[gid] = atan2(qy, qx) * a.inv_dlam;
  a.phi[gid] = atan2(qz, sqrt(qx * qx + qy * qy));
  a.lev[gid] = qk;
  a.move_m[gid] = last_m;
  a.move_k[gid] = last_k;
}

// ------------------------------------- line-search Newton departure search
// The reference's opt-in "newton_ls" solver (semilag/trajectory.py
// TRAJECTORY_SOLVERS, kernels.cu sl_departure_newton_ls_body): the same
// equation, gather and interpolant Jacobian, with each step accepted by a
// backtracking line search on the residual.  The interpolant is piecewise
// trilinear, so its Jacobian jumps at cell faces; where (dt/2)|J| nears one
// a full Newton step from one cell lands in the next, whose step points
// back, and the point cycles.  Here every iteration takes the Newton
// direction (or the residual itself where the 3 x 3 system is not solved:
// det(I - M) <= 0.05 or a pole) and halves it, at most four times, until
// the residual in grid cells falls by the Armijo factor 1 - 1e-4 alpha; the
// Newton step is capped at 20 times the residual.  A point whose residual
// is below 1e-4 cells stops.  The accepted trial point has been evaluated
// already, so an accepted full step costs one gather.  The reported move is
// the step AT THE RETURNED POINT (the linearised distance to the root, or
// the residual where the system was not solved), not the last move taken.
template <typename T>
struct NewtonEval {
  T res;           // |G(q) - q| in meridional grid cells (levels as they are)
  T de, dn, dk;    // the direction: Newton solve, or the residual itself
};

template <typename T>
__device__ __forceinline__ NewtonEval<T> newton_eval(const SlDepArgs<T>& a, T qx, T qy, T qz,
                                                     T qk, T ax, T ay, T az, int k, T ex, T ey,
                                                     T ez, T es, T c, T hdt, T klo, T khi,
                                                     T cells) {
  const T lam = atan2(qy, qx);
  const T rho = sqrt(qx * qx + qy * qy);
  const T phid = atan2(qz, rho);
  T w[4], dl[4], dp[4], dk[4];
  trilinear4_grad<T>(a, lam, phid, qk, w, dl, dp, dk);
  const T ux = ax - c * (ex + w[0]), uy = ay - c * (ey + w[1]), uz = az - c * (ez + w[2]);
  const T un = sqrt(ux * ux + uy * uy + uz * uz);
  const T px = ux / un, py = uy / un, pz = uz / un;
  const T pk_free = T(k) - hdt * (es + w[3]);
  const bool kheld = pk_free <= klo || pk_free >= khi;
  const T pk = min(max(pk_free, klo), khi);
  // local frame at q: east e, north nv
  const T cl = rho > T(0) ? qx / rho : T(1), sl = rho > T(0) ? qy / rho : T(0);
  const T cp = rho, sp = qz;
  const T e0 = -sl, e1 = cl;
  const T n0 = -sp * cl, n1 = -sp * sl, n2 = cp;
  const T dx = px - qx, dy = py - qy, dz = pz - qz;
  const T re = e0 * dx + e1 * dy, rn = n0 * dx + n1 * dy + n2 * dz, rk = pk - qk;
  NewtonEval<T> out{sqrt((re * re + rn * rn) * cells * cells + rk * rk), re, rn, rk};
  if (cp > T(1e-6)) {
    const T g = -c / un;
    const T icp = T(1) / cp;
    const T m00 = g * (e0 * dl[0] + e1 * dl[1]) * icp;
    const T m01 = g * (e0 * dp[0] + e1 * dp[1]);
    const T m02 = g * (e0 * dk[0] + e1 * dk[1]);
    const T m10 = g * (n0 * dl[0] + n1 * dl[1] + n2 * dl[2]) * icp;
    const T m11 = g * (n0 * dp[0] + n1 * dp[1] + n2 * dp[2]);
    const T m12 = g * (n0 * dk[0] + n1 * dk[1] + n2 * dk[2]);
    const T m20 = kheld ? T(0) : -hdt * dl[3] * icp;
    const T m21 = kheld ? T(0) : -hdt * dp[3];
    const T m22 = kheld ? T(0) : -hdt * dk[3];
    const T a00 = T(1) - m00, a01 = -m01, a02 = -m02;
    const T a10 = -m10, a11 = T(1) - m11, a12 = -m12;
    const T a20 = -m20, a21 = -m21, a22 = T(1) - m22;
    const T det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) +
                  a02 * (a10 * a21 - a11 * a20);
    if (isfinite(det) && det > T(0.05)) {
      const T id = T(1) / det;
      const T s0 = (re * (a11 * a22 - a12 * a21) - a01 * (rn * a22 - a12 * rk) +
                    a02 * (rn * a21 - a11 * rk)) * id;
      const T s1 = (a00 * (rn * a22 - a12 * rk) - re * (a10 * a22 - a12 * a20) +
                    a02 * (a10 * rk - rn * a20)) * id;
      const T s2 = (a00 * (a11 * rk - rn * a21) - a01 * (a10 * rk - rn * a20) +
                    re * (a10 * a21 - a11 * a20)) * id;
      if (isfinite(s0) && isfinite(s1) && isfinite(s2)) {
        const T step = sqrt((s0 * s0 + s1 * s1) * cells * cells + s2 * s2);
        const T ratio = step / (out.res + T(1e-30));
        const T shrink = ratio > T(20) ? T(20) / ratio : T(1);
        out.de = s0 * shrink;
        out.dn = s1 * shrink;
        out.dk = s2 * shrink;
      }
    }
  }
  return out;
}

template <typename T>
__global__ void __launch_bounds__(256) sl_departure_newton_ls_kernel(const SlDepArgs<T> a) {
  const int64_t n = (int64_t)a.nk * a.nja * a.ni;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int64_t gid = point_index(t, a.nk, a.nja, a.ni);
  const int plane = a.nja * a.ni;
  const int k = (int)(gid / plane);
  const int rem = (int)(gid - (int64_t)k * plane);
  const int j = rem / a.ni, i = rem - j * a.ni;
  const int64_t here = ((int64_t)k * a.njs + (j + a.lead)) * a.ni + i;
  const T lat = __ldg(a.lat_ext + a.ja0 + j + 2);
  const T lon = T((double)i * a.dlam);
  const T ax = cos(lat) * cos(lon), ay = cos(lat) * sin(lon), az = sin(lat);
  const T inv_r = T(1) / a.radius;
  const T dt = a.dt, hdt = T(0.5) * a.dt, c = hdt * inv_r;
  // the fixed-point search's first guess
  T qx = ax - dt * a.vx[here] * inv_r, qy = ay - dt * a.vy[here] * inv_r,
    qz = az - dt * a.vz[here] * inv_r;
  T nrm = sqrt(qx * qx + qy * qy + qz * qz);
  qx /= nrm; qy /= nrm; qz /= nrm;
  const T klo = T(-0.5), khi = T(a.nk) - T(0.5);
  T qk = min(max(T(k) - dt * a.sv[here], klo), khi);
  const T ex = a.vxe[gid], ey = a.vye[gid], ez = a.vze[gid], es = a.sve[gid];
  const T cells = T(a.nj) / T(2 * kHalfPi);  // meridional grid lengths per radian
  NewtonEval<T> cur = newton_eval<T>(a, qx, qy, qz, qk, ax, ay, az, k, ex, ey, ez, es, c, hdt,
                                     klo, khi, cells);
  for (int it = 0; it < a.iters && cur.res >= T(1e-4); ++it) {
    // q's local frame, in which the direction is expressed
    const T rho = sqrt(qx * qx + qy * qy);
    const T cl = rho > T(0) ? qx / rho : T(1), sl = rho > T(0) ? qy / rho : T(0);
    const T e0 = -sl, e1 = cl;
    const T n0 = -qz * cl, n1 = -qz * sl, n2 = rho;
    T alpha = T(1);
    T tx, ty, tz, tk;
    NewtonEval<T> trial;
    for (int ls = 0;; ++ls) {  // at most four halvings
      const T se = alpha * cur.de, sn = alpha * cur.dn;
      tx = qx + se * e0 + sn * n0;
      ty = qy + se * e1 + sn * n1;
      tz = qz + sn * n2;
      nrm = sqrt(tx * tx + ty * ty + tz * tz);
      tx /= nrm; ty /= nrm; tz /= nrm;
      tk = min(max(qk + alpha * cur.dk, klo), khi);
      trial = newton_eval<T>(a, tx, ty, tz, tk, ax, ay, az, k, ex, ey, ez, es, c, hdt, klo, khi,
                             cells);
      if (trial.res <= (T(1) - T(1e-4) * alpha) * cur.res || ls >= 4) break;
      alpha *= T(0.5);
    }
    qx = tx; qy = ty; qz = tz; qk = tk;
    cur = trial;
  }
  a.xi[gid] = atan2(qy, qx) * a.inv_dlam;
  a.phi[gid] = atan2(qz, sqrt(qx * qx + qy * qy));
  a.lev[gid] = qk;
  // the distance from the returned point to the root, linearised there
  a.move_m[gid] = a.radius * sqrt(cur.de * cur.de + cur.dn * cur.dn);
  a.move_k[gid] = fabs(cur.dk);
}

// ----------------------------------------------------------- tables
// The pole-extended table of one stencil width (semilag/tables.py:51-95,
// 164-217): G reflected rows each side, the data row and zonal shift each
// extended row reads, the reciprocal Lagrange denominators of every stencil
// start, and the bracket lookup (4 bins per extended row).
void build_width(SlWidth& w, const std::vector<double>& lat, int nlon, int NH) {
  const int nlat = (int)lat.size();
  const int G = NH / 2;  // 2 (cubic) or 3 (quintic)
  w.ghost = G;
  w.rows = nlat + 2 * G;
  w.lat_ext.assign(w.rows, 0.0);
  for (int g = 0; g < G; ++g) {
    w.lat_ext[G - 1 - g] = -kPi - lat[g];
    w.lat_ext[nlat + G + g] = kPi - lat[nlat - 1 - g];
  }
  for (int j = 0; j < nlat; ++j) w.lat_ext[G + j] = lat[j];
  for (int r = 1; r < w.rows; ++r)
    SHT_REQUIRE(w.lat_ext[r] > w.lat_ext[r - 1],
                "the pole-extended latitude table is not strictly ascending; the grid's "
                "outermost rings sit closer to a pole than the reflection of the rings inside "
                "them, which no Gaussian grid does and which the bracket search cannot represent");
  w.rowoff.resize(w.rows);
  w.rowshift.resize(w.rows);
  for (int r = 0; r < w.rows; ++r) {
    const int row = r - G;
    const int data = row < 0 ? -1 - row : (row >= nlat ? 2 * nlat - 1 - row : row);
    w.rowoff[r] = data * nlon;
    w.rowshift[r] = (row < 0 || row >= nlat) ? nlon / 2 : 0;
  }
  w.mrden.assign((size_t)(nlat + 1) * NH, 0.0);
  for (int s = 0; s <= nlat; ++s)
    for (int m = 0; m < NH; ++m) {
      double den = 1.0;
      for (int q = 0; q < NH; ++q)
        if (q != m) den *= w.lat_ext[s + m] - w.lat_ext[s + q];
      w.mrden[(size_t)s * NH + m] = 1.0 / den;
    }
  w.bins = 4 * w.rows;
  w.lut_scale = w.bins / kPi;
  w.mlut.resize(w.bins);
  const int lo = G - 1, hi = nlat + G - 1;  // bracket range of the width
  for (int b = 0; b < w.bins; ++b) {
    const double centre = -0.5 * kPi + (b + 0.5) / w.lut_scale;
    // searchsorted(lat_ext, centre, side="right") - 1
    const int m0 = (int)(std::upper_bound(w.lat_ext.begin(), w.lat_ext.end(), centre) -
                         w.lat_ext.begin()) - 1;
    w.mlut[b] = std::min(std::max(m0, lo), hi);
  }
}

template <typename T>
void upload_width(SlWidth& w) {
  std::vector<T> le(w.lat_ext.begin(), w.lat_ext.end()), md(w.mrden.begin(), w.mrden.end());
  SHT_CUDA_OR_THROW(cudaMalloc(&w.d_lat_ext, le.size() * sizeof(T)));
  SHT_CUDA_OR_THROW(cudaMalloc(&w.d_mrden, md.size() * sizeof(T)));
  SHT_CUDA_OR_THROW(cudaMalloc(&w.d_mlut, w.mlut.size() * sizeof(int32_t)));
  SHT_CUDA_OR_THROW(cudaMalloc(&w.d_rowoff, w.rowoff.size() * sizeof(int32_t)));
  SHT_CUDA_OR_THROW(cudaMalloc(&w.d_rowshift, w.rowshift.size() * sizeof(int32_t)));
  upload_now(w.d_lat_ext, le.data(), le.size() * sizeof(T));
  upload_now(w.d_mrden, md.data(), md.size() * sizeof(T));
  upload_now(w.d_mlut, w.mlut.data(), w.mlut.size() * sizeof(int32_t));
  upload_now(w.d_rowoff, w.rowoff.data(), w.rowoff.size() * sizeof(int32_t));
  upload_now(w.d_rowshift, w.rowshift.data(), w.rowshift.size() * sizeof(int32_t));
}

void free_width(SlWidth& w) {
  cudaFree(w.d_lat_ext);
  cudaFree(w.d_mrden);
  cudaFree(w.d_mlut);
  cudaFree(w.d_rowoff);
  cudaFree(w.d_rowshift);
  w.d_lat_ext = w.d_mrden = nullptr;
  w.d_mlut = w.d_rowoff = w.d_rowshift = nullptr;
}

const SlWidth& width_of(const sht_sl_tables* t, int order) {
  SHT_REQUIRE(order == 4 || order == 6,
              "the semi-Lagrangian gather's horizontal order must be one of 4, 6, got " +
                  std::to_string(order));
  if (order == 6)
    SHT_REQUIRE(t->w6.rows > 0, "the quintic gather needs six meridional rows and this grid has " +
                                    std::to_string(t->nlat) +
                                    "; the six-point tables were not built");
  return order == 6 ? t->w6 : t->w4;
}

template <typename T>
SlArgs<T> make_args(const sht_sl_tables* t, const SlWidth& w, const void* src, int64_t F,
                    int nlev, const void* xi, const void* phi, const void* lev, void* out,
                    void* cut) {
  SlArgs<T> a;
  a.src = (const T*)src;
  a.xi = (const T*)xi;
  a.phi = (const T*)phi;
  a.lev = (const T*)lev;
  a.lat_ext = (const T*)w.d_lat_ext;
  a.mrden = (const T*)w.d_mrden;
  a.mlut = w.d_mlut;
  a.rowoff = w.d_rowoff;
  a.rowshift = w.d_rowshift;
  a.out = (T*)out;
  a.cut = (T*)cut;
  a.F = (int)F;
  a.nk = nlev;
  a.nj = t->nlat;
  a.njs = a.nja = t->nlat;
  a.esc = nullptr;
  a.ni = t->nlon;
  a.nb = w.bins;
  a.lut_scale = (T)w.lut_scale;
  return a;
}

template <typename T, int NH>
void launch_gather(const SlArgs<T>& a, bool qm, bool def, cudaStream_t s) {
  const int64_t n = (int64_t)a.nk * a.nja * a.ni;
  const unsigned blocks = (unsigned)div_up(n, 256);
  if (qm && def)
    sl_gather_kernel<T, NH, true, true><<<blocks, 256, 0, s>>>(a);
  else if (qm)
    sl_gather_kernel<T, NH, true, false><<<blocks, 256, 0, s>>>(a);
  else
    sl_gather_kernel<T, NH, false, false><<<blocks, 256, 0, s>>>(a);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

void check_call(const sht_sl_tables* t, const void* src, int64_t fields, int nlev, const void* xi,
                const void* phi, const void* lev, const void* out) {
  SHT_REQUIRE(t != nullptr, "null semi-Lagrangian tables");
  SHT_REQUIRE(src && xi && phi && lev && out, "null array pointer");
  SHT_REQUIRE(fields >= 1 && fields <= (1 << 20), "fields must be in [1, 2^20]");
  SHT_REQUIRE(nlev >= 4, "a four-point vertical stencil needs nlev >= 4, got " +
                             std::to_string(nlev));
  const int64_t npts = (int64_t)nlev * t->nlat * t->nlon;
  SHT_REQUIRE(npts < ((int64_t)1 << 31) && fields * npts < ((int64_t)1 << 46),
              "the gather's volume is too large for one call");
  int dev = 0;
  SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
  SHT_REQUIRE(dev == t->device, "the tables live on another device");
}

}  // namespace
}  // namespace sht

using namespace sht;

extern "C" {

int sht_sl_tables_create(int nlat, int nlon, const double* lat_rad, const double* lon_rad,
                         int precision, sht_sl_tables** out) {
  return guarded([&] {
    SHT_REQUIRE(out != nullptr, "null output handle");
    *out = nullptr;
    SHT_REQUIRE(lat_rad != nullptr, "null latitude table");
    SHT_REQUIRE(precision == SHT_PREC_F64 || precision == SHT_PREC_F32,
                "the semi-Lagrangian gather is compiled for float32 and float64 only");
    SHT_REQUIRE(nlat >= 4, "a four-point meridional stencil needs nlat >= 4, got " +
                               std::to_string(nlat));
    SHT_REQUIRE(nlon >= 4 && nlon % 2 == 0,
                "nlon must be even so the polar reflection is an exact shift of nlon/2 columns, "
                "got " + std::to_string(nlon));
    std::vector<double> lat(lat_rad, lat_rad + nlat);
    for (int j = 1; j < nlat; ++j)
      SHT_REQUIRE(lat[j] > lat[j - 1],
                  "lat_rad must be strictly ascending; the bracket search and the pole "
                  "reflection both read it as a monotone table");
    if (lon_rad != nullptr) {
      const double dlam = 2.0 * kPi / nlon;
      double drift = 0.0;
      for (int i = 0; i < nlon; ++i) drift = std::max(drift, std::fabs(lon_rad[i] - i * dlam));
      SHT_REQUIRE(drift <= 1e-12,
                  "the zonal weights are the equispaced cubic Lagrange weights, which needs "
                  "lon[i] = i*2*pi/nlon");
    }
    auto* t = new sht_sl_tables;
    try {
      t->nlat = nlat;
      t->nlon = nlon;
      t->prec = precision;
      SHT_CUDA_OR_THROW(cudaGetDevice(&t->device));
      build_width(t->w4, lat, nlon, 4);
      if (nlat >= 6) build_width(t->w6, lat, nlon, 6);
      if (precision == SHT_PREC_F64) {
        upload_width<double>(t->w4);
        if (nlat >= 6) upload_width<double>(t->w6);
      } else {
        upload_width<float>(t->w4);
        if (nlat >= 6) upload_width<float>(t->w6);
      }
    } catch (...) {
      free_width(t->w4);
      free_width(t->w6);
      delete t;
      throw;
    }
    *out = t;
  });
}

int sht_sl_tables_destroy(sht_sl_tables* tables) {
  return guarded([&] {
    if (!tables) return;
    free_width(tables->w4);
    free_width(tables->w6);
    if (tables->d_lip) cudaFree(tables->d_lip);
    delete tables;
  });
}

int sht_sl_tables_read(const sht_sl_tables* tables, int order, double* lat_ext, double* mrden,
                       int32_t* mlut, int32_t* rowoff, int32_t* rowshift, int* rows, int* bins,
                       double* lut_scale) {
  return guarded([&] {
    SHT_REQUIRE(tables != nullptr, "null semi-Lagrangian tables");
    const SlWidth& w = width_of(tables, order);
    if (rows) *rows = w.rows;
    if (bins) *bins = w.bins;
    if (lut_scale) *lut_scale = w.lut_scale;
    if (lat_ext) std::copy(w.lat_ext.begin(), w.lat_ext.end(), lat_ext);
    if (mrden) std::copy(w.mrden.begin(), w.mrden.end(), mrden);
    if (mlut) std::copy(w.mlut.begin(), w.mlut.end(), mlut);
    if (rowoff) std::copy(w.rowoff.begin(), w.rowoff.end(), rowoff);
    if (rowshift) std::copy(w.rowshift.begin(), w.rowshift.end(), rowshift);
  });
}

static int departure_entry(int solver, const sht_sl_window* win, const sht_sl_tables* tables,
                           int nlev, const void* vx, const void* vy, const void* vz,
                           const void* level_rate, const void* vx_ex, const void* vy_ex,
                           const void* vz_ex, const void* level_rate_ex, int iterations,
                           double dt, double radius, void* xi, void* phi, void* level,
                           void* move_m, void* move_k, void* stream);

static int gather_entry(const sht_sl_window* win, const sht_sl_tables* tables, int order,
                        int limiter, int deficit, const void* src, int64_t fields, int nlev,
                        const void* xi, const void* phi, const void* level, void* out, void* cut,
                        void* stream) {
  return guarded([&] {
    check_call(tables, src, fields, nlev, xi, phi, level, out);
    SHT_REQUIRE(limiter == SHT_SL_NONE || limiter == SHT_SL_QUASI_MONOTONE,
                "the semi-Lagrangian gather's limiter must be one of 'quasi_monotone', 'none'");
    const SlWidth& w = width_of(tables, order);
    if (deficit) {
      SHT_REQUIRE(limiter != SHT_SL_NONE,
                  "the clip deficit is the mass the limiter moved, so an unlimited gather has "
                  "none to report; ask for a limiter or do not ask for the deficit");
      SHT_REQUIRE(order == 4, "the clip deficit is reported by the cubic gather only");
      SHT_REQUIRE(cut != nullptr, "null deficit array");
    }
    const bool qm = limiter == SHT_SL_QUASI_MONOTONE, def = deficit != 0;
    cudaStream_t s = (cudaStream_t)stream;
    auto band = [&](auto& a) {
      if (!win) return;
      a.rowoff = order == 6 ? win->d_rowoff6 : win->d_rowoff4;
      a.njs = win->s1 - win->s0;
      a.nja = win->a1 - win->a0;
      a.esc = win->d_esc;
    };
    if (tables->prec == SHT_PREC_F64) {
      auto a = make_args<double>(tables, w, src, fields, nlev, xi, phi, level, out, cut);
      band(a);
      if (order == 6) launch_gather<double, 6>(a, qm, false, s);
      else launch_gather<double, 4>(a, qm, def, s);
    } else {
      auto a = make_args<float>(tables, w, src, fields, nlev, xi, phi, level, out, cut);
      band(a);
      if (order == 6) launch_gather<float, 6>(a, qm, false, s);
      else launch_gather<float, 4>(a, qm, def, s);
    }
  });
}

int sht_sl_gather(const sht_sl_tables* tables, int order, int limiter, int deficit,
                  const void* src, int64_t fields, int nlev, const void* xi, const void* phi,
                  const void* level, void* out, void* cut, void* stream) {
  return gather_entry(nullptr, tables, order, limiter, deficit, src, fields, nlev, xi, phi, level,
                      out, cut, stream);
}

int sht_sl_window_create(const sht_sl_tables* tables, int s0, int s1, int a0, int a1,
                         sht_sl_window** out) {
  return guarded([&] {
    SHT_REQUIRE(out != nullptr, "null output handle");
    *out = nullptr;
    SHT_REQUIRE(tables != nullptr, "null semi-Lagrangian tables");
    const int nlat = tables->nlat;
    SHT_REQUIRE(0 <= s0 && s0 <= a0 && a0 < a1 && a1 <= s1 && s1 <= nlat,
                "a band window holds rows [" + std::to_string(s0) + ", " + std::to_string(s1) +
                    ") and computes rows [" + std::to_string(a0) + ", " + std::to_string(a1) +
                    "); the computed rows must lie inside the held rows and both inside the " +
                    std::to_string(nlat) + " rows of the grid");
    int dev = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
    SHT_REQUIRE(dev == tables->device, "the tables live on another device");
    auto rebase = [&](const SlWidth& w) {
      std::vector<int32_t> r(w.rowoff.size());
      for (size_t e = 0; e < r.size(); ++e) {
        const int row = w.rowoff[e] / tables->nlon;
        r[e] = (row >= s0 && row < s1) ? (row - s0) * tables->nlon : -1;
      }
      return r;
    };
    auto* h = new sht_sl_window;
    try {
      h->tables = tables;
      h->s0 = s0; h->s1 = s1; h->a0 = a0; h->a1 = a1;
      const auto r4 = rebase(tables->w4);
      SHT_CUDA_OR_THROW(cudaMalloc(&h->d_rowoff4, r4.size() * sizeof(int32_t)));
      upload_now(h->d_rowoff4, r4.data(), r4.size() * sizeof(int32_t));
      if (tables->w6.rows > 0) {
        const auto r6 = rebase(tables->w6);
        SHT_CUDA_OR_THROW(cudaMalloc(&h->d_rowoff6, r6.size() * sizeof(int32_t)));
        upload_now(h->d_rowoff6, r6.data(), r6.size() * sizeof(int32_t));
      }
      SHT_CUDA_OR_THROW(cudaMalloc(&h->d_esc, sizeof(int)));
      SHT_CUDA_OR_THROW(cudaMemset(h->d_esc, 0, sizeof(int)));
      SHT_CUDA_OR_THROW(cudaDeviceSynchronize());
    } catch (...) {
      cudaFree(h->d_rowoff4);
      cudaFree(h->d_rowoff6);
      cudaFree(h->d_esc);
      delete h;
      throw;
    }
    *out = h;
  });
}

int sht_sl_window_destroy(sht_sl_window* win) {
  return guarded([&] {
    if (!win) return;
    cudaFree(win->d_rowoff4);
    cudaFree(win->d_rowoff6);
    cudaFree(win->d_esc);
    delete win;
  });
}

int sht_sl_window_escape(sht_sl_window* win, int clear, int* escaped, void* stream) {
  return guarded([&] {
    SHT_REQUIRE(win != nullptr, "null band window");
    cudaStream_t s = (cudaStream_t)stream;
    if (escaped) {
      int flag = 0;
      SHT_CUDA_OR_THROW(cudaMemcpyAsync(&flag, win->d_esc, sizeof(int), cudaMemcpyDeviceToHost, s));
      SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
      *escaped = flag;
    }
    if (clear) SHT_CUDA_OR_THROW(cudaMemsetAsync(win->d_esc, 0, sizeof(int), s));
  });
}

int sht_sl_gather_band(const sht_sl_window* win, int order, int limiter, int deficit,
                       const void* src, int64_t fields, int nlev, const void* xi,
                       const void* phi, const void* level, void* out, void* cut, void* stream) {
  if (win == nullptr) {
    sht::set_error("null band window");
    return SHT_ERR_ARG;
  }
  return gather_entry(win, win->tables, order, limiter, deficit, src, fields, nlev, xi, phi,
                      level, out, cut, stream);
}

int sht_sl_departure_band(const sht_sl_window* win, int solver, int nlev, const void* vx,
                          const void* vy, const void* vz, const void* level_rate,
                          const void* vx_ex, const void* vy_ex, const void* vz_ex,
                          const void* level_rate_ex, int iterations, double dt, double radius,
                          void* xi, void* phi, void* level, void* move_m, void* move_k,
                          void* stream) {
  if (win == nullptr) {
    sht::set_error("null band window");
    return SHT_ERR_ARG;
  }
  return departure_entry(solver, win, win->tables, nlev, vx, vy, vz, level_rate, vx_ex,
                         vy_ex, vz_ex, level_rate_ex, iterations, dt, radius, xi, phi, level,
                         move_m, move_k, stream);
}

int sht_sl_gather_linear(const sht_sl_tables* tables, const void* src, int64_t fields, int nlev,
                         const void* xi, const void* phi, const void* level, void* out,
                         void* stream) {
  return guarded([&] {
    check_call(tables, src, fields, nlev, xi, phi, level, out);
    const SlWidth& w = tables->w4;
    const int64_t n = (int64_t)nlev * tables->nlat * tables->nlon;
    const unsigned blocks = (unsigned)div_up(n, 256);
    cudaStream_t s = (cudaStream_t)stream;
    if (tables->prec == SHT_PREC_F64) {
      auto a = make_args<double>(tables, w, src, fields, nlev, xi, phi, level, out, nullptr);
      sl_linear_kernel<double><<<blocks, 256, 0, s>>>(a);
    } else {
      auto a = make_args<float>(tables, w, src, fields, nlev, xi, phi, level, out, nullptr);
      sl_linear_kernel<float><<<blocks, 256, 0, s>>>(a);
    }
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

static int departure_entry(int solver, const sht_sl_window* win, const sht_sl_tables* tables,
                           int nlev, const void* vx,
                           const void* vy, const void* vz, const void* level_rate,
                           const void* vx_ex, const void* vy_ex, const void* vz_ex,
                           const void* level_rate_ex, int iterations, double dt, double radius,
                           void* xi, void* phi, void* level, void* move_m, void* move_k,
                           void* stream) {
  return guarded([&] {
    check_call(tables, vx, 1, nlev, vy, vz, level_rate, xi);
    SHT_REQUIRE(vx_ex && vy_ex && vz_ex && level_rate_ex && phi && level && move_m && move_k,
                "null array pointer");
    SHT_REQUIRE(iterations >= 1,
                "the departure-point search needs at least one iteration; zero would ship the "
                "explicit first guess, which is first order in dt and is not a trajectory");
    SHT_REQUIRE(std::isfinite(dt) && std::isfinite(radius) && radius > 0.0,
                "dt and radius must be finite, radius positive");
    const SlWidth& w = tables->w4;
    const int rows_out = win ? win->a1 - win->a0 : tables->nlat;
    const int64_t n = (int64_t)nlev * rows_out * tables->nlon;
    const unsigned blocks = (unsigned)div_up(n, 256);
    cudaStream_t s = (cudaStream_t)stream;
    auto fill = [&](auto* a) {
      using T = std::remove_cv_t<std::remove_pointer_t<decltype(a->vx)>>;
      a->vx = (const T*)vx; a->vy = (const T*)vy; a->vz = (const T*)vz;
      a->sv = (const T*)level_rate;
      a->vxe = (const T*)vx_ex; a->vye = (const T*)vy_ex; a->vze = (const T*)vz_ex;
      a->sve = (const T*)level_rate_ex;
      a->lat_ext = (const T*)w.d_lat_ext;
      a->mlut = w.d_mlut; a->rowoff = w.d_rowoff; a->rowshift = w.d_rowshift;
      a->xi = (T*)xi; a->phi = (T*)phi; a->lev = (T*)level;
      a->move_m = (T*)move_m; a->move_k = (T*)move_k;
      a->iters = iterations; a->nk = nlev; a->nj = tables->nlat; a->ni = tables->nlon;
      a->nb = w.bins;
      const double dlam = 2.0 * kPi / tables->nlon;
      a->dt = (T)dt; a->radius = (T)radius; a->dlam = dlam; a->inv_dlam = (T)(1.0 / dlam);
      a->lut_scale = (T)w.lut_scale;
      a->njs = a->nja = tables->nlat;
      a->ja0 = a->lead = 0;
      a->esc = nullptr;
      if (win) {
        a->rowoff = win->d_rowoff4;
        a->njs = win->s1 - win->s0;
        a->nja = win->a1 - win->a0;
        a->ja0 = win->a0;
        a->lead = win->a0 - win->s0;
        a->esc = win->d_esc;
      }
    };
    SHT_REQUIRE(solver >= kSolverFixedPoint && solver <= kSolverNewtonLs,
                "departure solver is 0 (fixed point), 1 (Newton) or 2 (line-search Newton)");
    if (tables->prec == SHT_PREC_F64) {
      SlDepArgs<double> a;
      fill(&a);
      if (solver == kSolverNewton) sl_departure_newton_kernel<double><<<blocks, 256, 0, s>>>(a);
      else if (solver == kSolverNewtonLs) sl_departure_newton_ls_kernel<double><<<blocks, 256, 0, s>>>(a);
      else sl_departure_kernel<double><<<blocks, 256, 0, s>>>(a);
    } else {
      SlDepArgs<float> a;
      fill(&a);
      if (solver == kSolverNewton) sl_departure_newton_kernel<float><<<blocks, 256, 0, s>>>(a);
      else if (solver == kSolverNewtonLs) sl_departure_newton_ls_kernel<float><<<blocks, 256, 0, s>>>(a);
      else sl_departure_kernel<float><<<blocks, 256, 0, s>>>(a);
    }
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

int sht_sl_departure(const sht_sl_tables* tables, int nlev, const void* vx, const void* vy,
                     const void* vz, const void* level_rate, const void* vx_ex,
                     const void* vy_ex, const void* vz_ex, const void* level_rate_ex,
                     int iterations, double dt, double radius, void* xi, void* phi,
                     void* level, void* move_m, void* move_k, void* stream) {
  return departure_entry(kSolverFixedPoint, nullptr, tables, nlev, vx, vy, vz, level_rate, vx_ex, vy_ex, vz_ex,
                         level_rate_ex, iterations, dt, radius, xi, phi, level, move_m, move_k,
                         stream);
}

int sht_sl_departure_newton(const sht_sl_tables* tables, int nlev, const void* vx,
                            const void* vy, const void* vz, const void* level_rate,
                            const void* vx_ex, const void* vy_ex, const void* vz_ex,
                            const void* level_rate_ex, int iterations, double dt, double radius,
                            void* xi, void* phi, void* level, void* move_m, void* move_k,
                            void* stream) {
  return departure_entry(kSolverNewton, nullptr, tables, nlev, vx, vy, vz, level_rate, vx_ex, vy_ex, vz_ex,
                         level_rate_ex, iterations, dt, radius, xi, phi, level, move_m, move_k,
                         stream);
}

int sht_sl_lipschitz(const sht_sl_tables* tables, int nlev, int a0, int a1, const void* vx,
                     const void* vy, const void* vz, const void* level_rate, int held0,
                     int held_rows, const void* vx_ex, const void* vy_ex, const void* vz_ex,
                     const void* level_rate_ex, int ex_held0, int ex_held_rows, double dt,
                     double radius, double reference_length, double* maxima, double* minima,
                     int64_t* argmin, void* stream) {
  return guarded([&] {
    SHT_REQUIRE(tables != nullptr, "null semi-Lagrangian tables");
    SHT_REQUIRE(vx && vy && vz && level_rate, "null wind array");
    SHT_REQUIRE(maxima && minima && argmin, "null result array");
    const bool has_ex = vx_ex != nullptr;
    SHT_REQUIRE(!has_ex || (vy_ex && vz_ex && level_rate_ex),
                "the extrapolated wind needs all four arrays (or none)");
    const int nlat = tables->nlat;
    SHT_REQUIRE(nlev >= 2, "the deformation diagnostic needs nlev >= 2");
    SHT_REQUIRE(0 <= a0 && a0 < a1 && a1 <= nlat, "arrival rows out of range");
    SHT_REQUIRE(std::isfinite(dt) && std::isfinite(radius) && radius > 0.0,
                "dt and radius must be finite, radius positive");
    SHT_REQUIRE(std::isfinite(reference_length) && reference_length > 0.0,
                "reference_length_m must be finite and positive");
    // Every row a derivative reads: the arrival rows and one neighbour each
    // side (the pole row itself beyond a pole).
    const int need0 = a0 == 0 ? 0 : a0 - 1, need1 = a1 == nlat ? nlat : a1 + 1;
    auto covers = [&](int h0, int rows) {
      return h0 >= 0 && rows >= 1 && h0 + rows <= nlat && h0 <= need0 && need1 <= h0 + rows;
    };
    SHT_REQUIRE(covers(held0, held_rows),
                "the deformation diagnostic reads a row the band's wind does not hold (halo "
                "escape)");
    SHT_REQUIRE(!has_ex || covers(ex_held0, ex_held_rows),
                "the deformation diagnostic reads a row the band's extrapolated wind does not "
                "hold (halo escape)");
    cudaStream_t s = (cudaStream_t)stream;
    if (!tables->d_lip) {
      void* p = nullptr;
      SHT_CUDA_OR_THROW(cudaMalloc(&p, lipschitz_scratch_bytes(nlat, tables->nlon)));
      const_cast<sht_sl_tables*>(tables)->d_lip = p;
    }
    LipResult r{};
    auto run = [&](auto zero) {
      using T = decltype(zero);
      LipFlow<T> w{{(const T*)vx, (const T*)vy, (const T*)vz, (const T*)level_rate}, held0,
                   held_rows};
      LipFlow<T> e{{nullptr, nullptr, nullptr, nullptr}, 0, 0};
      if (has_ex)
        e = LipFlow<T>{{(const T*)vx_ex, (const T*)vy_ex, (const T*)vz_ex, (const T*)level_rate_ex},
                       ex_held0, ex_held_rows};
      launch_lipschitz<T>(nlev, nlat, tables->nlon, a0, a1, (const T*)tables->w4.d_lat_ext, w, e,
                          dt, radius, reference_length, tables->d_lip, &r, s);
    };
    if (tables->prec == SHT_PREC_F64)
      run(0.0);
    else
      run(0.0f);
    for (int q = 0; q < 5; ++q) maxima[q] = r.maxima[q];
    minima[0] = r.minima[0];
    minima[1] = r.minima[1];
    argmin[0] = r.argmin[0];
    argmin[1] = r.argmin[1];
  });
}

int sht_sl_departure_newton_ls(const sht_sl_tables* tables, int nlev, const void* vx,
                               const void* vy, const void* vz, const void* level_rate,
                               const void* vx_ex, const void* vy_ex, const void* vz_ex,
                               const void* level_rate_ex, int iterations, double dt,
                               double radius, void* xi, void* phi, void* level, void* move_m,
                               void* move_k, void* stream) {
  return departure_entry(kSolverNewtonLs, nullptr, tables, nlev, vx, vy, vz, level_rate, vx_ex,
                         vy_ex, vz_ex, level_rate_ex, iterations, dt, radius, xi, phi, level,
                         move_m, move_k, stream);
}

}  // extern "C"
