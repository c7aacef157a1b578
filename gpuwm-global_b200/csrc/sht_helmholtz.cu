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
// (T+1, nlev, nlev) stack: four small mat-vecs per coefficient, with the
// operators held in shared memory by persistent CTAs and each thread
// accumulating four matrix rows against one 32-order column block.
#include "sht_plan.h"

namespace sht {
namespace {

template <typename T> using V2 = typename Vec2<T>::type;

constexpr int kMaxLev = 96;
constexpr int kRows = 6;                // matrix rows per thread per pass of a mat-vec
constexpr int kRowBlock = 8 * kRows;    // rows per pass over the CTA's 8 row groups

// Row stride of a shared matrix with `cols` columns and the vector length:
// a multiple of 4, so that four consecutive entries are one 16-byte (float)
// or two 16-byte (double) loads; padding entries are zero.
__host__ __device__ inline int padded(int cols) { return (cols + 3) & ~3; }
// Rows of a shared matrix: a multiple of one pass, padding rows zero.
__host__ __device__ inline int padded_rows(int rows) {
  return (rows + kRowBlock - 1) / kRowBlock * kRowBlock;
}

template <typename T> struct Quad;
template <> struct Quad<float> {
  static __device__ __forceinline__ void load(const float* p, float (&q)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
  }
};
template <> struct Quad<double> {
  static __device__ __forceinline__ void load(const double* p, double (&q)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
    q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y;
  }
};

// out[i] = f(i, sum_j M[i][j] * vec[j]) for rows i = ty + 8 r of every pass,
// column tx of the 32-column vector block.  M has padded_rows(rows) rows of
// padded(cols) entries and vec padded(cols) rows, all padding zero, so the
// loops carry no bounds tests; kRows rows share each loaded vector entry.
template <typename T, typename F>
__device__ __forceinline__ void matvec(const T* M, int rows, int cols, const V2<T>* vec, int tx,
                                       int ty, F&& finish) {
  const int ld = padded(cols);
  for (int i0 = 0; i0 < rows; i0 += kRowBlock) {
    T ar[kRows] = {}, ai[kRows] = {};
    const T* m0 = M + (i0 + ty) * ld;
    for (int j = 0; j < ld; j += 4) {
      V2<T> x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = vec[(j + u) * 32 + tx];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        T q[4];
        Quad<T>::load(m0 + 8 * r * ld + j, q);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          ar[r] += q[u] * x[u].x;
          ai[r] += q[u] * x[u].y;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r)
      if (i0 + ty + 8 * r < rows) finish(i0 + ty + 8 * r, ar[r], ai[r]);
  }
}

// Persistent: each CTA copies the five operators into shared memory once
// (rows padded to multiples of 4 with zeros) and then walks items (degree n,
// 32 consecutive orders), n fastest so that CTAs running together read
// neighbouring coefficient rows.  Items wholly above the triangle write zeros.
template <typename T>
__global__ void __launch_bounds__(256) helmholtz_kernel(int Tn, int nlev, double radius,
                                                        double tau, const T* __restrict__ mats,
                                                        const V2<T>* __restrict__ div,
                                                        const V2<T>* __restrict__ theta,
                                                        const V2<T>* __restrict__ lnps,
                                                        V2<T>* __restrict__ odiv,
                                                        V2<T>* __restrict__ otheta,
                                                        V2<T>* __restrict__ olnps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int L1 = nlev + 1;
  const int ldB = padded(L1), ldC = padded(nlev), ldV = padded(nlev), vp = padded(L1);
  T* sB = reinterpret_cast<T*>(smem_raw);  // nlev x L1
  T* sC = sB + padded_rows(nlev) * ldB;    // L1 x nlev
  T* sV = sC + padded_rows(L1) * ldC;      // nlev x nlev
  T* sVi = sV + padded_rows(nlev) * ldV;   // nlev x nlev
  T* sLam = sVi + padded_rows(nlev) * ldV; // nlev
  V2<T>* xs = reinterpret_cast<V2<T>*>(sLam + padded(nlev));  // [vp][32]
  V2<T>* fs = xs + vp * 32;                                   // [vp][32]
  V2<T>* gs = fs + vp * 32;                                   // [vp][32]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  {
    const T* B = mats;              // nlev x (nlev+1)
    const T* C = B + nlev * L1;     // (nlev+1) x nlev
    const T* V = C + L1 * nlev;     // nlev x nlev
    const T* Vi = V + nlev * nlev;  // nlev x nlev
    const T* lam = Vi + nlev * nlev;
    for (int e = tid; e < padded_rows(nlev) * ldB; e += 256) {
      const int i = e / ldB, j = e - i * ldB;
      sB[e] = (i < nlev && j < L1) ? B[i * L1 + j] : T(0);
    }
    for (int e = tid; e < padded_rows(L1) * ldC; e += 256) {
      const int i = e / ldC, j = e - i * ldC;
      sC[e] = (i < L1 && j < nlev) ? C[i * nlev + j] : T(0);
    }
    for (int e = tid; e < padded_rows(nlev) * ldV; e += 256) {
      const int i = e / ldV, j = e - i * ldV;
      const bool in = i < nlev && j < nlev;
      sV[e] = in ? V[i * nlev + j] : T(0);
      sVi[e] = in ? Vi[i * nlev + j] : T(0);
    }
    for (int e = tid; e < padded(nlev); e += 256) sLam[e] = e < nlev ? lam[e] : T(0);
    // Vector padding rows stay zero for the whole launch.
    for (int e = tid; e < 3 * vp * 32; e += 256) xs[e] = mk2<T>(T(0), T(0));
  }
  const int64_t t1 = Tn + 1;
  const int64_t lev = t1 * t1;  // one level of coefficients
  const int nmb = (Tn + 1 + 31) / 32;
  const T tw = T(tau);
  for (int item = blockIdx.x; item < nmb * (Tn + 1); item += gridDim.x) {
    const int mb = item / (Tn + 1);
    const int n = item - mb * (Tn + 1);
    const int m0 = mb * 32;
    const int m = m0 + tx;
    const bool live = m <= n;         // inside the triangle
    const int64_t cidx = n * t1 + m;  // (n, m) within one level
    if (m0 > n) {
      // Whole tile above the triangle: zeros.
      if (m <= Tn) {
        for (int i = ty; i < nlev; i += 8) {
          odiv[i * lev + cidx] = mk2<T>(T(0), T(0));
          otheta[i * lev + cidx] = mk2<T>(T(0), T(0));
        }
        if (ty == 0) olnps[cidx] = mk2<T>(T(0), T(0));
      }
      continue;
    }
    __syncthreads();  // the operators are staged; the previous item's vectors are consumed
    for (int i = ty; i < L1; i += 8) {
      V2<T> v = mk2<T>(T(0), T(0));
      if (live) v = i < nlev ? theta[i * lev + cidx] : lnps[cidx];
      xs[i * 32 + tx] = v;
    }
    __syncthreads();
    const T k2 = T((double)n * ((double)n + 1.0) / (radius * radius));
    // forcing = D + tau k2 (B x)
    matvec<T>(sB, nlev, L1, xs, tx, ty, [&](int i, T ar, T ai) {
      const V2<T> d = live ? div[i * lev + cidx] : mk2<T>(T(0), T(0));
      fs[i * 32 + tx] = mk2<T>(d.x + tw * k2 * ar, d.y + tw * k2 * ai);
    });
    __syncthreads();
    // g = diag(1/(1 + tau^2 k2 lambda)) V^-1 forcing
    matvec<T>(sVi, nlev, nlev, fs, tx, ty, [&](int i, T ar, T ai) {
      const T modal = T(1) / (T(1) + (tw * tw * k2) * sLam[i]);
      gs[i * 32 + tx] = mk2<T>(ar * modal, ai * modal);
    });
    __syncthreads();
    // D' = V g  (into fs, and out)
    matvec<T>(sV, nlev, nlev, gs, tx, ty, [&](int i, T ar, T ai) {
      V2<T> dn = mk2<T>(ar, ai);
      if (n == 0) dn = live ? div[i * lev + cidx] : dn;  // degree zero passes through
      if (m == 0) dn.y = T(0);
      if (!live) dn = mk2<T>(T(0), T(0));
      fs[i * 32 + tx] = dn;
      if (m <= Tn) odiv[i * lev + cidx] = dn;
    });
    __syncthreads();
    // x' = x + tau C D'
    matvec<T>(sC, L1, nlev, fs, tx, ty, [&](int i, T ar, T ai) {
      const V2<T> x = xs[i * 32 + tx];
      V2<T> xn = mk2<T>(x.x + tw * ar, x.y + tw * ai);
      if (n == 0) xn = x;
      if (m == 0) xn.y = T(0);
      if (!live) xn = mk2<T>(T(0), T(0));
      if (m <= Tn) {
        if (i < nlev)
          otheta[i * lev + cidx] = xn;
        else
          olnps[cidx] = xn;
      }
    });
  }
}

}  // namespace

template <typename T>
void launch_helmholtz(const sht_plan* p, int nlev, const T* mats, double tau_w, const T* div,
                      const T* theta, const T* lnps, T* odiv, T* otheta, T* olnps,
                      cudaStream_t s) {
  SHT_REQUIRE(nlev >= 1 && nlev <= kMaxLev, "nlev must be in [1, 96]");
  const int L1 = nlev + 1;
  const size_t mat_elems = (size_t)padded_rows(nlev) * padded(L1) +
                           (size_t)padded_rows(L1) * padded(nlev) +
                           2 * (size_t)padded_rows(nlev) * padded(nlev) + padded(nlev);
  const size_t sm = sizeof(T) * mat_elems + sizeof(V2<T>) * 32 * (size_t)(3 * padded(L1));
  SHT_CUDA_OR_THROW(cudaFuncSetAttribute(helmholtz_kernel<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int per_sm = 0, dev = 0, sms = 0;
  SHT_CUDA_OR_THROW(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, helmholtz_kernel<T>, 256, sm));
  SHT_REQUIRE(per_sm > 0, "Helmholtz kernel does not fit on an SM");
  SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
  SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t items = div_up(p->T + 1, 32) * (int64_t)(p->T + 1);
  const int ctas = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  helmholtz_kernel<T><<<ctas, dim3(32, 8), sm, s>>>(
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
