// The reference's Fourier waist, (*lead, nlat, T+1) complex, in and out of
// the folded waist the engine's kernels use.
//
// The reference names the buffer between its longitude FFT and its Legendre
// contraction (FourierWaist, src/arwen_global/spectral/transform.py:417-629)
// so that callers can fill it a latitude band at a time and drain it the
// same way (fourier_waist, contract_waist, contract_to_waist, waist_to_grid,
// transform.py:1294-1404, 1435-1452, 1629-1716).  The engine keeps its
// waist folded at the equator: per order m and latitude pair h (row h and
// its mirror row nlat-1-h) the symmetric and antisymmetric combinations
// S and D, plane rows innermost.  These two kernels convert:
//
//   export (folded -> reference):  X(h) = c (S + D),  X(mirror) = c (S - D)
//   import (reference -> folded):  S = c (X(h) + X(mirror)),  D = c (X(h) - X(mirror))
//
// with c = 1/2 or 1 by the convention of the kernel on the folded side (the
// longitude FFT's fold sums the two rows, the inverse FFT's unfold adds and
// subtracts S and D), and the equator row of an odd nlat kept once (X = S,
// D = 0).  A 32 (orders) x 32 (planes) shared tile turns the folded side's
// plane-contiguous rows into the reference side's order-contiguous rows.
#include "sht_plan.h"

namespace sht {
namespace {

template <typename T> using V2 = typename Vec2<T>::type;

template <typename T>
__global__ void __launch_bounds__(256) waist_export_kernel(int Tn, int H, int nlat, int nlat_odd,
                                                           double c, int zonal,
                                                           const V2<T>* __restrict__ wf,
                                                           int64_t planes, V2<T>* __restrict__ out) {
  __shared__ V2<T> tile[2][32][33];  // [side][plane][order]
  const int m0 = blockIdx.x * 32;
  const int h = blockIdx.y;
  const int64_t p0 = (int64_t)blockIdx.z * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int t1 = Tn + 1;
  const bool eq = nlat_odd && h == H - 1;
  const T cc = T(c);
  for (int mm = ty; mm < 32; mm += 8) {
    const int m = m0 + mm;
    const int64_t p = p0 + tx;
    V2<T> a = mk2<T>(T(0), T(0)), b = a;
    if (m < t1 && p < planes) {
      const V2<T> S = wf[((int64_t)(m * 2 + 0) * H + h) * planes + p];
      const V2<T> D = wf[((int64_t)(m * 2 + 1) * H + h) * planes + p];
      if (eq) {
        a = S;
      } else {
        a = mk2<T>(cc * (S.x + D.x), cc * (S.y + D.y));
        b = mk2<T>(cc * (S.x - D.x), cc * (S.y - D.y));
      }
      if (zonal) {  // i m X
        const T mf = T(m);
        a = mk2<T>(-mf * a.y, mf * a.x);
        b = mk2<T>(-mf * b.y, mf * b.x);
      }
    }
    tile[0][tx][mm] = a;
    tile[1][tx][mm] = b;
  }
  __syncthreads();
  for (int pp = ty; pp < 32; pp += 8) {
    const int64_t p = p0 + pp;
    const int m = m0 + tx;
    if (p >= planes || m >= t1) continue;
    out[(p * nlat + h) * t1 + m] = tile[0][pp][tx];
    if (!eq) out[(p * nlat + (nlat - 1 - h)) * t1 + m] = tile[1][pp][tx];
  }
}

// `fields` F > 1: the input is a stack of F fields of planes / F planes each
// (field-major, the reference's stacked (u, v) waist), written with the
// fields interleaved per plane (column plane * F + field), the layout the
// multi-field contractions and their epilogues read.
template <typename T>
__global__ void __launch_bounds__(256) waist_import_kernel(int Tn, int H, int nlat, int nlat_odd,
                                                           double c, const V2<T>* __restrict__ in,
                                                           int64_t planes, int fields,
                                                           V2<T>* __restrict__ wf,
                                                           float* __restrict__ rowmax) {
  __shared__ V2<T> tile[2][32][33];  // [S/D][plane][order]
  __shared__ float red[2][8][32];
  const int m0 = blockIdx.x * 32;
  const int h = blockIdx.y;
  const int64_t p0 = (int64_t)blockIdx.z * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int t1 = Tn + 1;
  const bool eq = nlat_odd && h == H - 1;
  const T cc = T(c);
  for (int pp = ty; pp < 32; pp += 8) {
    const int64_t p = p0 + pp;
    const int m = m0 + tx;
    V2<T> S = mk2<T>(T(0), T(0)), D = S;
    if (p < planes && m < t1) {
      const V2<T> x0 = in[(p * nlat + h) * t1 + m];
      if (eq) {
        S = x0;
      } else {
        const V2<T> x1 = in[(p * nlat + (nlat - 1 - h)) * t1 + m];
        S = mk2<T>(cc * (x0.x + x1.x), cc * (x0.y + x1.y));
        D = mk2<T>(cc * (x0.x - x1.x), cc * (x0.y - x1.y));
      }
    }
    tile[0][pp][tx] = S;
    tile[1][pp][tx] = D;
  }
  __syncthreads();
  float mre = 0.f, mim = 0.f;
  const int64_t p = p0 + tx;
  const int64_t per_field = planes / fields;
  const int64_t col = fields == 1 ? p : (p % per_field) * fields + p / per_field;
  for (int mm = ty; mm < 32; mm += 8) {
    const int m = m0 + mm;
    if (m >= t1 || p >= planes) continue;
    const V2<T> S = tile[0][tx][mm], D = tile[1][tx][mm];
    wf[((int64_t)(m * 2 + 0) * H + h) * planes + col] = S;
    wf[((int64_t)(m * 2 + 1) * H + h) * planes + col] = D;
    mre = fmaxf(mre, fmaxf((float)fabs(S.x), (float)fabs(D.x)));
    mim = fmaxf(mim, fmaxf((float)fabs(S.y), (float)fabs(D.y)));
  }
  if (rowmax != nullptr) {
    red[0][ty][tx] = mre;
    red[1][ty][tx] = mim;
    __syncthreads();
    if (ty == 0 && p < planes) {
      float ra = 0.f, rb = 0.f;
      for (int k = 0; k < 8; ++k) {
        ra = fmaxf(ra, red[0][k][tx]);
        rb = fmaxf(rb, red[1][k][tx]);
      }
      atomicMax(reinterpret_cast<int*>(rowmax + 2 * col), __float_as_int(ra));
      atomicMax(reinterpret_cast<int*>(rowmax + 2 * col + 1), __float_as_int(rb));
    }
  }
}

}  // namespace

template <typename T>
void launch_waist_export(const sht_plan* p, const T* wfold, int64_t planes, double c, int zonal,
                         T* waist, cudaStream_t s) {
  if (planes == 0) return;
  dim3 grid((unsigned)div_up(p->T + 1, 32), (unsigned)p->H, (unsigned)div_up(planes, 32));
  SHT_REQUIRE(grid.z <= 65535, "too many planes for one waist launch");
  waist_export_kernel<T><<<grid, dim3(32, 8), 0, s>>>(p->T, p->H, p->nlat, p->nlat_odd ? 1 : 0, c,
                                                      zonal, (const V2<T>*)wfold, planes,
                                                      (V2<T>*)waist);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template <typename T>
void launch_waist_import(const sht_plan* p, const T* waist, int64_t planes, double c, T* wfold,
                         float* rowmax, cudaStream_t s, int fields) {
  if (planes == 0) return;
  SHT_REQUIRE(fields >= 1 && planes % fields == 0, "waist import: planes not a multiple of fields");
  dim3 grid((unsigned)div_up(p->T + 1, 32), (unsigned)p->H, (unsigned)div_up(planes, 32));
  SHT_REQUIRE(grid.z <= 65535, "too many planes for one waist launch");
  waist_import_kernel<T><<<grid, dim3(32, 8), 0, s>>>(p->T, p->H, p->nlat, p->nlat_odd ? 1 : 0, c,
                                                      (const V2<T>*)waist, planes, fields,
                                                      (V2<T>*)wfold, rowmax);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

#define INST(T)                                                                                  \
  template void launch_waist_export<T>(const sht_plan*, const T*, int64_t, double, int, T*,     \
                                       cudaStream_t);                                           \
  template void launch_waist_import<T>(const sht_plan*, const T*, int64_t, double, T*, float*,  \
                                       cudaStream_t, int);
INST(float)
INST(double)
#undef INST

}  // namespace sht
