// Per-degree semi-implicit stage solve in the vertical-mode basis.
//
// VerticalModeSemiImplicit.solve_shifted (src/arwen_global/semi_implicit.py:
// 921-953): with x = (theta, ln ps) and k_n^2 = n(n+1)/a^2,
//   forcing = D + tau k^2 (B x)
//   D'      = (I + tau^2 k^2 M)^-1 forcing = V diag(1/(1 + tau^2 k^2 lambda)) V^-1 forcing
//   x'      = x + tau C D'
// then degree zero passes through and the outputs are projected (_finish,
// semi_implicit.py:815-843).  The inverse is applied modally
// (helmholtz_inverse, semi_implicit.py:585-609) instead of as a stored
// (T+1, nlev, nlev) stack: three small mat-vecs per coefficient.  One CTA
// handles one degree n and 32 consecutive orders; the level vectors live in
// shared memory and every warp reads one matrix row at a time (broadcast).
#include "sht_plan.h"

namespace sht {
namespace {

template <typename T> using V2 = typename Vec2<T>::type;

constexpr int kMaxLev = 96;

template <typename T>
__global__ void helmholtz_kernel(int Tn, int nlev, double radius, double tau,
                                 const T* __restrict__ mats, const V2<T>* __restrict__ div,
                                 const V2<T>* __restrict__ theta, const V2<T>* __restrict__ lnps,
                                 V2<T>* __restrict__ odiv, V2<T>* __restrict__ otheta,
                                 V2<T>* __restrict__ olnps) {
  extern __shared__ unsigned char smem_raw[];
  V2<T>* xs = reinterpret_cast<V2<T>*>(smem_raw);  // [nlev+1][32]
  V2<T>* fs = xs + (nlev + 1) * 32;                 // [nlev][32]
  V2<T>* gs = fs + nlev * 32;                       // [nlev][32]
  const int n = blockIdx.y;
  const int m0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m = m0 + tx;
  const int64_t t1 = Tn + 1;
  const int L1 = nlev + 1;
  const T* B = mats;                    // nlev x (nlev+1)
  const T* C = B + nlev * L1;           // (nlev+1) x nlev
  const T* V = C + L1 * nlev;           // nlev x nlev
  const T* Vi = V + nlev * nlev;        // nlev x nlev
  const T* lam = Vi + nlev * nlev;      // nlev
  const bool live = m <= n;             // inside the triangle
  const int64_t cidx = n * t1 + m;      // (n, m) within one level

  if (m0 > Tn) return;
  if (m0 > n) {
    // Whole tile above the triangle: zeros.
    for (int i = ty; i < nlev; i += blockDim.y) {
      if (m <= Tn) {
        odiv[i * t1 * t1 + cidx] = mk2<T>(T(0), T(0));
        otheta[i * t1 * t1 + cidx] = mk2<T>(T(0), T(0));
      }
    }
    if (ty == 0 && m <= Tn) olnps[cidx] = mk2<T>(T(0), T(0));
    return;
  }
  for (int i = ty; i < L1; i += blockDim.y) {
    V2<T> v = mk2<T>(T(0), T(0));
    if (live) v = i < nlev ? theta[i * t1 * t1 + cidx] : lnps[cidx];
    xs[i * 32 + tx] = v;
  }
  __syncthreads();
  const T k2 = T((double)n * ((double)n + 1.0) / (radius * radius));
  const T tw = T(tau);
  // forcing = D + tau k2 (B x)
  for (int i = ty; i < nlev; i += blockDim.y) {
    T ar = 0, ai = 0;
    for (int j = 0; j < L1; ++j) {
      T b = B[i * L1 + j];
      V2<T> x = xs[j * 32 + tx];
      ar += b * x.x;
      ai += b * x.y;
    }
    V2<T> d = live ? div[i * t1 * t1 + cidx] : mk2<T>(T(0), T(0));
    fs[i * 32 + tx] = mk2<T>(d.x + tw * k2 * ar, d.y + tw * k2 * ai);
  }
  __syncthreads();
  // g = diag(1/(1 + tau^2 k2 lambda)) V^-1 forcing
  for (int i = ty; i < nlev; i += blockDim.y) {
    T ar = 0, ai = 0;
    for (int j = 0; j < nlev; ++j) {
      T v = Vi[i * nlev + j];
      V2<T> f = fs[j * 32 + tx];
      ar += v * f.x;
      ai += v * f.y;
    }
    T modal = T(1) / (T(1) + (tw * tw * k2) * lam[i]);
    gs[i * 32 + tx] = mk2<T>(ar * modal, ai * modal);
  }
  __syncthreads();
  // D' = V g  (stored back into fs)
  for (int i = ty; i < nlev; i += blockDim.y) {
    T ar = 0, ai = 0;
    for (int j = 0; j < nlev; ++j) {
      T v = V[i * nlev + j];
      V2<T> g = gs[j * 32 + tx];
      ar += v * g.x;
      ai += v * g.y;
    }
    V2<T> dn = mk2<T>(ar, ai);
    if (n == 0) dn = live ? div[i * t1 * t1 + cidx] : dn;  // degree zero passes through
    if (m == 0) dn.y = T(0);
    if (!live) dn = mk2<T>(T(0), T(0));
    fs[i * 32 + tx] = dn;
  }
  __syncthreads();
  // x' = x + tau C D'
  for (int i = ty; i < L1; i += blockDim.y) {
    T ar = 0, ai = 0;
    for (int j = 0; j < nlev; ++j) {
      T c = C[i * nlev + j];
      V2<T> d = fs[j * 32 + tx];
      ar += c * d.x;
      ai += c * d.y;
    }
    V2<T> x = xs[i * 32 + tx];
    V2<T> xn = mk2<T>(x.x + tw * ar, x.y + tw * ai);
    if (n == 0) xn = x;
    if (m == 0) xn.y = T(0);
    if (!live) xn = mk2<T>(T(0), T(0));
    if (m <= Tn) {
      if (i < nlev)
        otheta[i * t1 * t1 + cidx] = xn;
      else
        olnps[cidx] = xn;
    }
  }
  for (int i = ty; i < nlev; i += blockDim.y)
    if (m <= Tn) odiv[i * t1 * t1 + cidx] = fs[i * 32 + tx];
}

}  // namespace

template <typename T>
void launch_helmholtz(const sht_plan* p, int nlev, const T* mats, double tau_w, const T* div,
                      const T* theta, const T* lnps, T* odiv, T* otheta, T* olnps,
                      cudaStream_t s) {
  SHT_REQUIRE(nlev >= 1 && nlev <= kMaxLev, "nlev must be in [1, 96]");
  size_t sm = sizeof(V2<T>) * 32 * (size_t)(3 * nlev + 1);
  SHT_CUDA_OR_THROW(cudaFuncSetAttribute(helmholtz_kernel<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)std::max<size_t>(sm, 48 * 1024)));
  dim3 grid((unsigned)div_up(p->T + 1, 32), (unsigned)(p->T + 1));
  helmholtz_kernel<T><<<grid, dim3(32, 8), sm, s>>>(
      p->T, nlev, p->radius, tau_w, mats, (const V2<T>*)div, (const V2<T>*)theta,
      (const V2<T>*)lnps, (V2<T>*)odiv, (V2<T>*)otheta, (V2<T>*)olnps);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template void launch_helmholtz<float>(const sht_plan*, int, const float*, double, const float*,
                                      const float*, const float*, float*, float*, float*,
                                      cudaStream_t);
template void launch_helmholtz<double>(const sht_plan*, int, const double*, double, const double*,
                                       const double*, const double*, double*, double*, double*,
                                       cudaStream_t);

}  // namespace sht
