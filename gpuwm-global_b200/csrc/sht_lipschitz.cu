// The trajectory deformation diagnostics of the semi-Lagrangian step: the
// flow Jacobian at every arrival point, the norms the reference reports and
// the fold determinants its gate reads (the reference's
// semilag/trajectory.py:1174-1420, numpy specification 1038-1171, the
// derivatives 672-752).
//
// Per point (level k, row j, lon i), from the Cartesian wind (vx, vy, vz)
// and the level rate s:
//   d/dx = (f[i+1] - f[i-1]) / (2 dlam) / (a max(cos phi, 1e-12)),
//   d/dy = the three-point formula on the non-uniform latitudes, the rows
//          beyond a pole being the pole row half a turn round, / a,
//   d/dk = centred in the level index, one-sided at the ends;
// the Jacobian projected on the local east/north basis (the vertical entries
// scaled by a reference length L), its Frobenius norm, the spectral norms of
// the 2 x 2 horizontal block, of the whole 3 x 3 and of the "balanced" 3 x 3
// (coupling blocks rescaled to their geometric mean) through the closed-form
// top eigenvalue of J^T J, and det(I + c J) with c = +dt/2 (departure side,
// the wind) and c = -dt/2 (arrival side, the extrapolated wind).
//
// The arithmetic is the reference's numpy expressions in the same order and
// without fused multiply-adds (every product and sum rounded on its own), so
// the only differences from the reference are the last bits of sin, cos and
// acos.  One thread per point, consecutive threads along a latitude row (the
// neighbour loads of a warp share cache lines), one resident wave of CTAs
// (three per SM in FP32 at 78 registers, two in FP64); each CTA reduces its
// points to partial maxima/minima in shared memory and one CTA combines the
// partials.  Every field is read from DRAM about once, but the kernel is
// bound by its arithmetic (some 45 correctly rounded divisions, 10 square
// roots and two arccosines per point), not by those 32 bytes per point.
#include <algorithm>
#include <cfloat>
#include <climits>

#include "sht_lipschitz.h"

namespace sht {
namespace {

// Products and sums that the compiler may not fuse.
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

template <typename T> struct Eps;
template <> struct Eps<float> { static constexpr float v = FLT_EPSILON; };
template <> struct Eps<double> { static constexpr double v = DBL_EPSILON; };

constexpr int kLipThreads = 256;
constexpr int kLipBlocksPerSm = 4;
constexpr int kLipMaxBlocks = 160 * kLipBlocksPerSm;

template <typename T>
struct LipArgs {
  int nlev, nlat, nlon, a0, nrows;
  LipFlow<T> wind, ex;  // ex.f[0] == nullptr: the arrival side reads the wind
  const T* lat_ext;
  double dlam;
  T two_dlam, radius, inv_y, lref, half;
  T* part;              // [gridDim.x][7]
  long long* part_idx;  // [gridDim.x][2]
  // Per arrival row: sin phi, cos phi, 1 / (a max(cos phi, 1e-12)) and the
  // three-point latitude formula's numerators and denominators n0, d0, n1,
  // d1, n2, d2; per longitude: sin lam, cos lam.  Filled once per launch by
  // lipschitz_tables_kernel with the very operations a point would do.
  T* rows;  // [nrows][kRowVals]
  T* cols;  // [nlon][2]
};

constexpr int kRowVals = 9;

// The twelve derivatives of one flow at one point: d/dx, d/dy, d/dk of the
// three Cartesian components, then of the level rate.
template <typename T>
struct Grad {
  T vx[3], vy[3], vk[3];  // [component]
  T sx, sy, sk;
};

template <typename T>
__device__ __forceinline__ T at(const LipFlow<T>& F, int c, int nlon, int nheld, int k, int j,
                                int i) {
  return __ldg(F.f[c] + ((int64_t)k * nheld + (j - F.held0)) * nlon + i);
}

template <typename T>
__global__ void lipschitz_tables_kernel(LipArgs<T> a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.nrows) {
    const int j = a.a0 + t;
    const T lat = __ldg(a.lat_ext + j + 2);
    const T sph = sin(lat), cph = cos(lat);
    const T x0 = __ldg(a.lat_ext + j + 1), x1 = lat, x2 = __ldg(a.lat_ext + j + 3);
    T* r = a.rows + (int64_t)t * kRowVals;
    r[0] = sph;
    r[1] = cph;
    r[2] = T(1) / mul(a.radius, fmax(cph, T(1e-12)));
    r[3] = sub(x1, x2);
    r[4] = mul(sub(x0, x1), sub(x0, x2));
    r[5] = sub(sub(mul(T(2), x1), x0), x2);
    r[6] = mul(sub(x1, x0), sub(x1, x2));
    r[7] = sub(x1, x0);
    r[8] = mul(sub(x2, x0), sub(x2, x1));
  }
  if (t < a.nlon) {
    const T lon = (T)((double)t * a.dlam);
    a.cols[2 * t] = sin(lon);
    a.cols[2 * t + 1] = cos(lon);
  }
}

template <typename T>
__device__ void gradient(const LipArgs<T>& a, const LipFlow<T>& F, int k, int j, int i, T inv_x,
                         const T* __restrict__ row, Grad<T>& g) {
  const int nlon = a.nlon, nh = F.held;
  const int ip = i + 1 == nlon ? 0 : i + 1;
  const int im = i == 0 ? nlon - 1 : i - 1;
  // the row beyond a pole: the pole row itself, read half a turn round
  const int half_turn = (i - nlon / 2 + nlon) % nlon;
  const int ju = j == 0 ? 0 : j - 1, iu = j == 0 ? half_turn : i;
  const int jd = j == a.nlat - 1 ? j : j + 1, id = j == a.nlat - 1 ? half_turn : i;
  const T n0 = row[3], d0 = row[4], n1 = row[5], d1 = row[6], n2 = row[7], d2 = row[8];
  const int kd = k == 0 ? 0 : k - 1, ku = k == a.nlev - 1 ? k : k + 1;
  const bool centred = k > 0 && k < a.nlev - 1;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const T dx = mul(inv_x, sub(at(F, c, nlon, nh, k, j, ip), at(F, c, nlon, nh, k, j, im)) / a.two_dlam);
    const T f0 = at(F, c, nlon, nh, k, ju, iu), f1 = at(F, c, nlon, nh, k, j, i),
            f2 = at(F, c, nlon, nh, k, jd, id);
    const T dy = mul(a.inv_y, add(add(mul(f0, n0) / d0, mul(f1, n1) / d1), mul(f2, n2) / d2));
    const T up = at(F, c, nlon, nh, ku, j, i), dn = at(F, c, nlon, nh, kd, j, i);
    const T dk = centred ? mul(T(0.5), sub(up, dn)) : sub(up, dn);
    if (c < 3) {
      g.vx[c] = dx;
      g.vy[c] = dy;
      g.vk[c] = dk;
    } else {
      g.sx = dx;
      g.sy = dy;
      g.sk = dk;
    }
  }
}

// Largest eigenvalue of a symmetric 3 x 3, scaled to unit trace, by the
// trigonometric solution of its characteristic cubic (trajectory.py:621-663).
template <typename T>
__device__ T sym3_top(T a00, T a01, T a02, T a11, T a12, T a22) {
  const T tiny = Eps<T>::v;
  const T trace = add(add(a00, a11), a22);
  const T scale = fmax(trace, tiny);
  const T inv = T(1) / scale;
  a00 = mul(a00, inv); a01 = mul(a01, inv); a02 = mul(a02, inv);
  a11 = mul(a11, inv); a12 = mul(a12, inv); a22 = mul(a22, inv);
  const T q = add(add(a00, a11), a22) / T(3);
  const T b00 = sub(a00, q), b11 = sub(a11, q), b22 = sub(a22, q);
  const T off = add(add(mul(a01, a01), mul(a02, a02)), mul(a12, a12));
  const T p2 = add(add(add(mul(b00, b00), mul(b11, b11)), mul(b22, b22)), mul(T(2), off)) / T(6);
  const T p = sqrt(fmax(p2, T(0)));
  const T safe = fmax(p, tiny);
  const T det = add(sub(mul(b00, sub(mul(b11, b22), mul(a12, a12))),
                        mul(a01, sub(mul(a01, b22), mul(a12, a02)))),
                    mul(a02, sub(mul(a01, a12), mul(b11, a02))));
  T r = det / mul(mul(mul(T(2), safe), safe), safe);
  r = fmin(fmax(r, T(-1)), T(1));
  const T phi = acos(r) / T(3);
  return mul(scale, add(q, mul(mul(T(2), p), cos(phi))));
}

// The local basis: east (-sin lam, cos lam, 0), north (-sin phi cos lam,
// -sin phi sin lam, cos phi); a vector's east and north components.
template <typename T>
struct Basis {
  T exx, exy, eyx, eyy, eyz;
  __device__ T east(const T (&v)[3]) const { return add(mul(exx, v[0]), mul(exy, v[1])); }
  __device__ T north(const T (&v)[3]) const {
    return add(add(mul(eyx, v[0]), mul(eyy, v[1])), mul(eyz, v[2]));
  }
};

// det(I + c J) of the flow Jacobian (trajectory.py:1140-1171).
template <typename T>
__device__ T fold_det(const Basis<T>& b, const Grad<T>& g, T c) {
  const T m00 = add(T(1), mul(c, b.east(g.vx)));
  const T m01 = mul(c, b.east(g.vy));
  const T m02 = mul(c, b.east(g.vk));
  const T m10 = mul(c, b.north(g.vx));
  const T m11 = add(T(1), mul(c, b.north(g.vy)));
  const T m12 = mul(c, b.north(g.vk));
  const T m20 = mul(c, g.sx), m21 = mul(c, g.sy), m22 = add(T(1), mul(c, g.sk));
  return add(sub(mul(m00, sub(mul(m11, m22), mul(m12, m21))),
                 mul(m01, sub(mul(m10, m22), mul(m12, m20)))),
             mul(m02, sub(mul(m10, m21), mul(m11, m20))));
}

// Norms of the Jacobian (trajectory.py:1038-1097): spectral (mixed units,
// length L), Frobenius, horizontal block, balanced.
template <typename T>
__device__ void jacobian_norms(const Basis<T>& b, const Grad<T>& g, T lref, T (&out)[4]) {
  const T j00 = b.east(g.vx), j01 = b.east(g.vy), j02 = b.east(g.vk) / lref;
  const T j10 = b.north(g.vx), j11 = b.north(g.vy), j12 = b.north(g.vk) / lref;
  const T j20 = mul(lref, g.sx), j21 = mul(lref, g.sy), j22 = g.sk;
  T fr = mul(j00, j00);
  fr = add(fr, mul(j01, j01));
  fr = add(fr, mul(j02, j02));
  fr = add(fr, mul(j10, j10));
  fr = add(fr, mul(j11, j11));
  fr = add(fr, mul(j12, j12));
  fr = add(fr, mul(j20, j20));
  fr = add(fr, mul(j21, j21));
  fr = add(fr, mul(j22, j22));
  const T h00 = add(mul(j00, j00), mul(j10, j10));
  const T h11 = add(mul(j01, j01), mul(j11, j11));
  const T h01 = add(mul(j00, j01), mul(j10, j11));
  const T dh = sub(h00, h11);
  const T rad = sqrt(fmax(add(mul(T(0.25), mul(dh, dh)), mul(h01, h01)), T(0)));
  const T horizontal = sqrt(fmax(add(mul(T(0.5), add(h00, h11)), rad), T(0)));
  const T spectral = sqrt(fmax(
      sym3_top<T>(add(h00, mul(j20, j20)), add(add(mul(j00, j01), mul(j10, j11)), mul(j20, j21)),
                  add(add(mul(j00, j02), mul(j10, j12)), mul(j20, j22)),
                  add(h11, mul(j21, j21)), add(add(mul(j01, j02), mul(j11, j12)), mul(j21, j22)),
                  add(add(mul(j02, j02), mul(j12, j12)), mul(j22, j22))),
      T(0)));
  // the coupling blocks rescaled to the geometric mean of their magnitudes
  const T e0 = mul(j02, lref), e1 = mul(j12, lref);
  const T d0 = g.sx, d1 = g.sy;
  const T emag = sqrt(add(mul(e0, e0), mul(e1, e1)));
  const T dmag = sqrt(add(mul(d0, d0), mul(d1, d1)));
  const T gmean = sqrt(mul(emag, dmag));
  const T se = emag > T(0) ? gmean / emag : T(0);
  const T sd = dmag > T(0) ? gmean / dmag : T(0);
  const T c02 = mul(e0, se), c12 = mul(e1, se), c20 = mul(d0, sd), c21 = mul(d1, sd);
  const T balanced = sqrt(fmax(
      sym3_top<T>(add(h00, mul(c20, c20)), add(add(mul(j00, j01), mul(j10, j11)), mul(c20, c21)),
                  add(add(mul(j00, c02), mul(j10, c12)), mul(c20, j22)),
                  add(h11, mul(c21, c21)), add(add(mul(j01, c02), mul(j11, c12)), mul(c21, j22)),
                  add(add(mul(c02, c02), mul(c12, c12)), mul(j22, j22))),
      T(0)));
  out[0] = spectral;
  out[1] = sqrt(fr);
  out[2] = horizontal;
  out[3] = balanced;
}

// A candidate minimum replaces the current one when it is smaller, or equal
// and earlier; NaN never replaces.
template <typename T>
__device__ __forceinline__ void take_min(T v, long long idx, T& cur, long long& cur_idx) {
  if (v < cur || (v == cur && idx < cur_idx)) {
    cur = v;
    cur_idx = idx;
  }
}

template <typename T>
__global__ void __launch_bounds__(kLipThreads, sizeof(T) == 4 ? 3 : 2) lipschitz_kernel(LipArgs<T> a) {
  T mx[5] = {T(0), T(0), T(0), T(0), T(0)};
  T mn[2] = {T(INFINITY), T(INFINITY)};
  long long at_mn[2] = {LLONG_MAX, LLONG_MAX};
  const long long npts = (long long)a.nlev * a.nrows * a.nlon;
  const T cplus = a.half, cminus = -a.half;
  // The grid stride and the first point decomposed into (level, row, lon)
  // once; each step then carries the lon and row components by one
  // subtraction at most (the stride's own components are below nlon and
  // nrows), so the loop does no integer division per point.
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long plane = (long long)a.nrows * a.nlon;
  const int step_i = (int)(stride % a.nlon), step_r = (int)((stride / a.nlon) % a.nrows);
  const int step_k = (int)(stride / plane);
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i = (int)(p % a.nlon), r = (int)((p / a.nlon) % a.nrows);
  int k = (int)(p / plane);
  for (; p < npts; p += stride) {
    const int j = a.a0 + r;
    const T* row = a.rows + (int64_t)r * kRowVals;
    const T sph = row[0], cph = row[1], inv_x = row[2];
    const T sla = a.cols[2 * i], cla = a.cols[2 * i + 1];
    const Basis<T> b{-sla, cla, mul(-sph, cla), mul(-sph, sla), cph};
    Grad<T> g;
    gradient<T>(a, a.wind, k, j, i, inv_x, row, g);
    T nr[4];
    jacobian_norms<T>(b, g, a.lref, nr);
    const T vert = fabs(g.sk);
    const T v5[5] = {nr[0], nr[1], nr[2], vert, nr[3]};
#pragma unroll
    for (int q = 0; q < 5; ++q) mx[q] = v5[q] > mx[q] ? v5[q] : mx[q];
    take_min(fold_det<T>(b, g, cplus), p, mn[0], at_mn[0]);
    if (a.ex.f[0] != nullptr) gradient<T>(a, a.ex, k, j, i, inv_x, row, g);
    take_min(fold_det<T>(b, g, cminus), p, mn[1], at_mn[1]);
    i += step_i;
    int carry = 0;
    if (i >= a.nlon) {
      i -= a.nlon;
      carry = 1;
    }
    r += step_r + carry;
    carry = 0;
    if (r >= a.nrows) {
      r -= a.nrows;
      carry = 1;
    }
    k += step_k + carry;
  }
  // CTA reduction through shared memory, then one partial record per CTA.
  __shared__ T s_v[7][kLipThreads];
  __shared__ long long s_i[2][kLipThreads];
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 5; ++q) s_v[q][t] = mx[q];
  s_v[5][t] = mn[0];
  s_v[6][t] = mn[1];
  s_i[0][t] = at_mn[0];
  s_i[1][t] = at_mn[1];
  __syncthreads();
  for (int st = kLipThreads / 2; st > 0; st >>= 1) {
    if (t < st) {
#pragma unroll
      for (int q = 0; q < 5; ++q) s_v[q][t] = s_v[q][t + st] > s_v[q][t] ? s_v[q][t + st] : s_v[q][t];
#pragma unroll
      for (int q = 0; q < 2; ++q) take_min(s_v[5 + q][t + st], s_i[q][t + st], s_v[5 + q][t], s_i[q][t]);
    }
    __syncthreads();
  }
  if (t == 0) {
#pragma unroll
    for (int q = 0; q < 7; ++q) a.part[blockIdx.x * 7 + q] = s_v[q][0];
    a.part_idx[blockIdx.x * 2 + 0] = s_i[0][0];
    a.part_idx[blockIdx.x * 2 + 1] = s_i[1][0];
  }
}

// One CTA combines the partial records of n CTAs into the result record
// (7 values in double, then 2 indices) at `out`.
template <typename T>
__global__ void __launch_bounds__(kLipThreads) lipschitz_combine_kernel(const T* part,
                                                                        const long long* part_idx,
                                                                        int n, double* out,
                                                                        long long* out_idx) {
  __shared__ T s_v[7][kLipThreads];
  __shared__ long long s_i[2][kLipThreads];
  const int t = threadIdx.x;
  T mx[5] = {T(0), T(0), T(0), T(0), T(0)};
  T mn[2] = {T(INFINITY), T(INFINITY)};
  long long at_mn[2] = {LLONG_MAX, LLONG_MAX};
  for (int b = t; b < n; b += kLipThreads) {
#pragma unroll
    for (int q = 0; q < 5; ++q) mx[q] = part[b * 7 + q] > mx[q] ? part[b * 7 + q] : mx[q];
#pragma unroll
    for (int q = 0; q < 2; ++q) take_min(part[b * 7 + 5 + q], part_idx[b * 2 + q], mn[q], at_mn[q]);
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) s_v[q][t] = mx[q];
  s_v[5][t] = mn[0];
  s_v[6][t] = mn[1];
  s_i[0][t] = at_mn[0];
  s_i[1][t] = at_mn[1];
  __syncthreads();
  for (int st = kLipThreads / 2; st > 0; st >>= 1) {
    if (t < st) {
#pragma unroll
      for (int q = 0; q < 5; ++q) s_v[q][t] = s_v[q][t + st] > s_v[q][t] ? s_v[q][t + st] : s_v[q][t];
#pragma unroll
      for (int q = 0; q < 2; ++q) take_min(s_v[5 + q][t + st], s_i[q][t + st], s_v[5 + q][t], s_i[q][t]);
    }
    __syncthreads();
  }
  if (t == 0) {
#pragma unroll
    for (int q = 0; q < 7; ++q) out[q] = (double)s_v[q][0];
    out_idx[0] = s_i[0][0];
    out_idx[1] = s_i[1][0];
  }
}

}  // namespace

// Scratch layout: partials (7 doubles + 2 indices per CTA), the result
// record (7 doubles, 2 indices), then the row and column tables in doubles.
constexpr size_t kPartBytes = (size_t)kLipMaxBlocks * (7 * sizeof(double) + 2 * sizeof(long long));
constexpr size_t kResultBytes = 7 * sizeof(double) + 2 * sizeof(long long);

size_t lipschitz_scratch_bytes(int nlat, int nlon) {
  return kPartBytes + kResultBytes + sizeof(double) * ((size_t)nlat * kRowVals + 2 * (size_t)nlon);
}

template <typename T>
void launch_lipschitz(int nlev, int nlat, int nlon, int a0, int a1, const T* lat_ext,
                      const LipFlow<T>& wind, const LipFlow<T>& ex, double dt_s,
                      double radius_m, double reference_length_m, void* scratch,
                      LipResult* out, cudaStream_t s) {
  int dev = 0, sms = 0;
  SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
  SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int per_sm = 0;
  SHT_CUDA_OR_THROW(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lipschitz_kernel<T>, kLipThreads, 0));
  per_sm = std::max(1, std::min(per_sm, kLipBlocksPerSm));
  const long long npts = (long long)nlev * (a1 - a0) * nlon;
  const int blocks = (int)std::max<long long>(
      1, std::min<long long>({(npts + kLipThreads - 1) / kLipThreads, (long long)sms * per_sm,
                              (long long)kLipMaxBlocks}));
  LipArgs<T> a;
  a.nlev = nlev;
  a.nlat = nlat;
  a.nlon = nlon;
  a.a0 = a0;
  a.nrows = a1 - a0;
  a.wind = wind;
  a.ex = ex;
  a.lat_ext = lat_ext;
  a.dlam = 2.0 * kPi / nlon;
  a.two_dlam = (T)(2.0 * a.dlam);
  a.radius = (T)radius_m;
  a.inv_y = (T)(1.0 / radius_m);
  a.lref = (T)reference_length_m;
  a.half = (T)(0.5 * dt_s);
  // scratch: [kLipMaxBlocks][7] T partials, [kLipMaxBlocks][2] indices, the
  // 7 reduced doubles and 2 reduced indices
  char* base = static_cast<char*>(scratch);
  a.part = reinterpret_cast<T*>(base);
  a.part_idx = reinterpret_cast<long long*>(base + (size_t)kLipMaxBlocks * 7 * sizeof(double));
  double* res = reinterpret_cast<double*>(base + kPartBytes);
  long long* res_idx = reinterpret_cast<long long*>(res + 7);
  a.rows = reinterpret_cast<T*>(base + kPartBytes + kResultBytes);
  a.cols = a.rows + (size_t)a.nrows * kRowVals;
  const int nt = std::max(a.nrows, nlon);
  lipschitz_tables_kernel<T><<<(nt + 255) / 256, 256, 0, s>>>(a);
  SHT_CUDA_OR_THROW(cudaGetLastError());
  lipschitz_kernel<T><<<blocks, kLipThreads, 0, s>>>(a);
  SHT_CUDA_OR_THROW(cudaGetLastError());
  lipschitz_combine_kernel<T><<<1, kLipThreads, 0, s>>>(a.part, a.part_idx, blocks, res, res_idx);
  SHT_CUDA_OR_THROW(cudaGetLastError());
  double host[7];
  long long host_idx[2];
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(host, res, sizeof(host), cudaMemcpyDeviceToHost, s));
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(host_idx, res_idx, sizeof(host_idx), cudaMemcpyDeviceToHost, s));
  SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
  for (int q = 0; q < 5; ++q) out->maxima[q] = host[q];
  out->minima[0] = host[5];
  out->minima[1] = host[6];
  out->argmin[0] = host_idx[0];
  out->argmin[1] = host_idx[1];
}

template void launch_lipschitz<float>(int, int, int, int, int, const float*, const LipFlow<float>&,
                                      const LipFlow<float>&, double, double, double, void*,
                                      LipResult*, cudaStream_t);
template void launch_lipschitz<double>(int, int, int, int, int, const double*,
                                       const LipFlow<double>&, const LipFlow<double>&, double,
                                       double, double, void*, LipResult*, cudaStream_t);

}  // namespace sht
