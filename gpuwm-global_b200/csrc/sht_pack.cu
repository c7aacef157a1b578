// Spectral-side layout kernels.
//
// pack:   coefficients (planes, T+1, T+1) [n, m] -> the synthesis operand
//         Cfold, rows (m, q, i) with n = m + q + 2i and the (plane, field,
//         re/im) columns innermost; optional per-degree factor (the inverse
//         Laplacian of the vector synthesis, transform.py:1804-1811).
// unpack: the analysis output Cfold -> coefficients, zero above the
//         triangle and Imag(c[n,0]) = 0 (transform.py:1435-1452); the vector
//         mode combines the rotational and shear contractions into
//         (vorticity, divergence) with the i*m factor and projects
//         (vector.py:113-134).
// Both go through a 32 x 32 shared tile so the [n, m] side is read/written
// along m and the folded side along the plane index.
#include "sht_plan.h"

namespace sht {
namespace {

template <typename T> using V2 = typename Vec2<T>::type;

// Row base of order m in the folded operand Cfold (orders below m fill
// sum_{m' < m} (T + 1 - m') rows); with size0 the size of its parity-0
// block, row(m, q, i) = base + (q ? size0 : 0) + i.
__device__ __forceinline__ int64_t cf_base(int T, int m) {
  return (int64_t)m * (T + 1) - (int64_t)m * (m - 1) / 2;
}

// One CTA: 32 orders x NB degrees x 32 planes.  All NB x 4 loads of a thread
// are issued before the CTA's one barrier, and the row maxima are merged over
// the whole block before one atomic per column.  INVLAP: divide by the
// Laplacian eigenvalue -n(n+1)/a^2 (zero at degree 0, Imag = 0 at m = 0).
template <typename T> struct PackCfg { static constexpr int NB = sizeof(T) == 4 ? 4 : 2; };

template <typename T, bool INVLAP>
__global__ void __launch_bounds__(256) pack_kernel(int Tn, double radius,
                                                   const V2<T>* __restrict__ c0,
                                                   const V2<T>* __restrict__ c1, int64_t planes,
                                                   int F, V2<T>* __restrict__ cf,
                                                   float* __restrict__ rowmax) {
  constexpr int NB = PackCfg<T>::NB;
  __shared__ V2<T> tile[NB][32][33];
  __shared__ float red[2][8][32];
  const int m0 = blockIdx.x * 32;
  const int n0 = blockIdx.y * NB;
  if (m0 > n0 + NB - 1 || n0 > Tn) return;  // the whole block is above the triangle
  const int f = blockIdx.z % F;
  const int64_t p0 = (int64_t)(blockIdx.z / F) * 32;
  const V2<T>* src = f ? c1 : c0;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t t1 = Tn + 1;
  {
    const int m = m0 + tx;
    V2<T> v[NB][4];
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
      const int n = n0 + nb;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int64_t p = p0 + ty + 8 * k;
        v[nb][k] = mk2<T>(T(0), T(0));
        if (p < planes && n <= Tn && m <= n) v[nb][k] = __ldcs(src + (p * t1 + n) * t1 + m);
      }
    }
#pragma unroll
    for (int nb = 0; nb < NB; ++nb)
#pragma unroll
      for (int k = 0; k < 4; ++k) tile[nb][ty + 8 * k][tx] = v[nb][k];
  }
  __syncthreads();
  const int64_t Rc = planes * F;
  const int64_t p = p0 + tx;
  float mre = 0.f, mim = 0.f;
  if (p < planes) {
    V2<T>* col = cf + p * F + f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int m = m0 + ty + 8 * k;
      if (m > Tn) break;
      const int64_t base = cf_base(Tn, m);
      const int size0 = parity_count(Tn, m, 0);
#pragma unroll
      for (int nb = 0; nb < NB; ++nb) {
        const int n = n0 + nb;
        if (n > Tn || m > n) continue;
        const int q = (n - m) & 1, i = (n - m) >> 1;
        V2<T> v = tile[nb][tx][ty + 8 * k];
        if constexpr (INVLAP) {
          const T eig = T(-((double)n * ((double)n + 1.0)) / (radius * radius));
          // c / eig (complex by real), zero at degree 0
          v = n == 0 ? mk2<T>(T(0), T(0)) : mk2<T>(v.x / eig, v.y / eig);
          if (m == 0) v.y = T(0);  // project() inside inverse_laplacian
        }
        col[(base + (q ? size0 : 0) + i) * Rc] = v;
        mre = fmaxf(mre, (float)fabs(v.x));
        mim = fmaxf(mim, (float)fabs(v.y));
      }
    }
  }
  if (rowmax != nullptr) {
    // Row maxima of this CTA's 32 columns: reduce the 8 ty groups, publish once.
    red[0][ty][tx] = mre;
    red[1][ty][tx] = mim;
    __syncthreads();
    if (ty == 0 && p < planes) {
      float ra = 0.f, rb = 0.f;
      for (int k = 0; k < 8; ++k) {
        ra = fmaxf(ra, red[0][k][tx]);
        rb = fmaxf(rb, red[1][k][tx]);
      }
      const int64_t col = p * F + f;
      atomicMax(reinterpret_cast<int*>(rowmax + 2 * col), __float_as_int(ra));
      atomicMax(reinterpret_cast<int*>(rowmax + 2 * col + 1), __float_as_int(rb));
    }
  }
}

// One CTA: 32 orders x NB degrees x 32 planes, every load issued before the
// CTA's one barrier; a CTA wholly above the triangle writes zeros only.
template <typename T, int MODE> struct UnpackCfg {
  static constexpr int NO = MODE == kUnpackVorDiv ? 2 : 1;  // output fields
  static constexpr int NB = sizeof(T) == 4 ? 2 : 1;
};

template <typename T, int MODE>
__global__ void __launch_bounds__(256) unpack_kernel(int Tn, const V2<T>* __restrict__ cf0,
                                                     const V2<T>* __restrict__ cf1, int64_t planes,
                                                     V2<T>* __restrict__ o0, V2<T>* __restrict__ o1) {
  constexpr int NB = UnpackCfg<T, MODE>::NB, NO = UnpackCfg<T, MODE>::NO;
  __shared__ V2<T> tile[NO][NB][32][33];
  const int m0 = blockIdx.x * 32;
  const int n0 = blockIdx.y * NB;
  const int64_t p0 = (int64_t)blockIdx.z * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t t1 = Tn + 1;
  const V2<T> zero = mk2<T>(T(0), T(0));
  if (m0 > n0 + NB - 1) {
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
      const int n = n0 + nb;
      if (n > Tn) break;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int64_t pl = p0 + ty + 8 * k;
        const int m = m0 + tx;
        if (pl >= planes || m > Tn) continue;
        const int64_t off = (pl * t1 + n) * t1 + m;
        o0[off] = zero;
        if (NO == 2) o1[off] = zero;
      }
    }
    return;
  }
  const int64_t Rc = planes * NO;
  const int64_t p = p0 + tx;
  {
    V2<T> va[NB][4], vb[NB][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int m = m0 + ty + 8 * k;
      const int64_t base = m <= Tn ? cf_base(Tn, m) : 0;
      const int size0 = m <= Tn ? parity_count(Tn, m, 0) : 0;
#pragma unroll
      for (int nb = 0; nb < NB; ++nb) {
        const int n = n0 + nb;
        va[nb][k] = zero;
        vb[nb][k] = zero;
        if (n <= Tn && m <= n && p < planes) {
          const int q = (n - m) & 1, i = (n - m) >> 1;
          const int64_t row = base + (q ? size0 : 0) + i;
          if constexpr (MODE == kUnpackScalar) {
            va[nb][k] = __ldcs(cf0 + row * Rc + p);
          } else if constexpr (MODE == kUnpackDiv) {
            // cf0: rotational rows of u, cf1: shear rows of v (one column per plane).
            const V2<T> ru = __ldcs(cf0 + row * Rc + p), sv = __ldcs(cf1 + row * Rc + p);
            const T mf = T(m);
            va[nb][k] = mk2<T>(-mf * ru.y - sv.x, mf * ru.x - sv.y);
          } else {
            // rot/shear rows hold (u, v) per plane: columns 2p (u), 2p+1 (v).
            const V2<T> ru = __ldcs(cf0 + row * Rc + 2 * p), rv = __ldcs(cf0 + row * Rc + 2 * p + 1);
            const V2<T> su = __ldcs(cf1 + row * Rc + 2 * p), sv = __ldcs(cf1 + row * Rc + 2 * p + 1);
            const T mf = T(m);
            // zeta = i m rot[v] + shear[u];  D = i m rot[u] - shear[v]
            va[nb][k] = mk2<T>(-mf * rv.y + su.x, mf * rv.x + su.y);
            vb[nb][k] = mk2<T>(-mf * ru.y - sv.x, mf * ru.x - sv.y);
          }
          if (m == 0) {
            va[nb][k].y = T(0);
            vb[nb][k].y = T(0);
          }
        }
      }
    }
#pragma unroll
    for (int nb = 0; nb < NB; ++nb)
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        tile[0][nb][tx][ty + 8 * k] = va[nb][k];
        if (NO == 2) tile[NO - 1][nb][tx][ty + 8 * k] = vb[nb][k];
      }
  }
  __syncthreads();
#pragma unroll
  for (int nb = 0; nb < NB; ++nb) {
    const int n = n0 + nb;
    if (n > Tn) break;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int pp = ty + 8 * k;
      const int64_t pl = p0 + pp;
      const int m = m0 + tx;
      if (pl >= planes || m > Tn) continue;
      const int64_t off = (pl * t1 + n) * t1 + m;
      // Above the triangle the tile holds zeros.
      o0[off] = tile[0][nb][pp][tx];
      if (NO == 2) o1[off] = tile[NO - 1][nb][pp][tx];
    }
  }
}

template <typename T>
__global__ void elementwise_kernel(int Tn, double radius, int mode, const V2<T>* __restrict__ in,
                                   int64_t total, V2<T>* __restrict__ out) {
  const int64_t t1 = Tn + 1;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    int m = (int)(idx % t1);
    int n = (int)((idx / t1) % t1);
    V2<T> v = in[idx];
    T eig = T(-((double)n * ((double)n + 1.0)) / (radius * radius));
    if (mode == kElemLaplacian) {
      v = mk2<T>(v.x * eig, v.y * eig);
    } else {
      if (mode == kElemInvLaplacian) v = n == 0 ? mk2<T>(T(0), T(0)) : mk2<T>(v.x / eig, v.y / eig);
      if (m > n) v = mk2<T>(T(0), T(0));
      if (m == 0) v.y = T(0);
    }
    out[idx] = v;
  }
}

}  // namespace

template <typename T>
void launch_pack(const sht_plan* p, const T* coeff0, const T* coeff1, int64_t planes, int mode,
                 T* cfold, cudaStream_t s, float* rowmax) {
  if (planes == 0) return;
  int F = coeff1 ? 2 : 1;
  dim3 grid((unsigned)div_up(p->T + 1, 32), (unsigned)div_up(p->T + 1, PackCfg<T>::NB),
            (unsigned)(div_up(planes, 32) * F));
  SHT_REQUIRE(grid.z <= 65535, "too many planes for one pack launch");
  if (mode == kPackInvLap)
    pack_kernel<T, true><<<grid, dim3(32, 8), 0, s>>>(p->T, p->radius, (const V2<T>*)coeff0,
                                                      (const V2<T>*)coeff1, planes, F,
                                                      (V2<T>*)cfold, rowmax);
  else
    pack_kernel<T, false><<<grid, dim3(32, 8), 0, s>>>(p->T, p->radius, (const V2<T>*)coeff0,
                                                       (const V2<T>*)coeff1, planes, F,
                                                       (V2<T>*)cfold, rowmax);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template <typename T, int MODE>
void launch_unpack_mode(const sht_plan* p, const T* cf0, const T* cf1, int64_t planes, T* out0,
                        T* out1, cudaStream_t s) {
  dim3 grid((unsigned)div_up(p->T + 1, 32), (unsigned)div_up(p->T + 1, UnpackCfg<T, MODE>::NB),
            (unsigned)div_up(planes, 32));
  SHT_REQUIRE(grid.z <= 65535, "too many planes for one unpack launch");
  unpack_kernel<T, MODE><<<grid, dim3(32, 8), 0, s>>>(p->T, (const V2<T>*)cf0, (const V2<T>*)cf1,
                                                      planes, (V2<T>*)out0, (V2<T>*)out1);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template <typename T>
void launch_unpack(const sht_plan* p, int mode, const T* cf0, const T* cf1, int64_t planes,
                   T* out0, T* out1, cudaStream_t s) {
  if (planes == 0) return;
  if (mode == kUnpackVorDiv)
    launch_unpack_mode<T, kUnpackVorDiv>(p, cf0, cf1, planes, out0, out1, s);
  else if (mode == kUnpackDiv)
    launch_unpack_mode<T, kUnpackDiv>(p, cf0, cf1, planes, out0, out1, s);
  else
    launch_unpack_mode<T, kUnpackScalar>(p, cf0, cf1, planes, out0, out1, s);
}

template <typename T>
void launch_elementwise(const sht_plan* p, int mode, const T* in, int64_t planes, T* out,
                        cudaStream_t s) {
  int64_t total = planes * (int64_t)(p->T + 1) * (p->T + 1);
  if (total == 0) return;
  int blocks = (int)std::min<int64_t>(div_up(total, 256), 148 * 16);
  elementwise_kernel<T><<<blocks, 256, 0, s>>>(p->T, p->radius, mode, (const V2<T>*)in, total,
                                               (V2<T>*)out);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

#define INST(T)                                                                                  \
  template void launch_pack<T>(const sht_plan*, const T*, const T*, int64_t, int, T*,          \
                               cudaStream_t, float*);                                           \
  template void launch_unpack<T>(const sht_plan*, int, const T*, const T*, int64_t, T*, T*,    \
                                 cudaStream_t);                                                 \
  template void launch_elementwise<T>(const sht_plan*, int, const T*, int64_t, T*, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace sht
