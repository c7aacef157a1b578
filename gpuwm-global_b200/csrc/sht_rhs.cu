// Fused right-hand-side kernels of the dycore step: the elementwise chains
// that consume the synthesis output (the reference's spectral/fused.py:233-386
// CuPy kernels and their numpy specifications in dynamics.py:1355-1490,
// 1575-1610).
//
//   momentum_bernoulli  av = zeta + f;  pf = R Tv pg;
//                       mu = av v - wu - pf ge;  mv = -av u - wv - pf gn;
//                       bern = 0.5 (u^2 + v^2) + phi
//                       (f, ge, gn horizontal fields broadcast over levels)
//   tracer_flux         m = dp s;  fx = m u;  fy = m v
//   scalar_tendency     out = (-h - vert - s dpt) / dp
//   vertical_flux_divergence
//                       van Leer limited upstream flux through every
//                       interface, out[k] = F[k+1] - F[k], F[0] = F[nlev] = 0
//
// Leading (tracer) axes: s, h, vert and the outputs of the last three may
// hold B blocks of (nlev, nlat, nlon); dp, u, v, dpt, w, pf, ph are one
// block, shared.  The arithmetic follows the specifications' association.
//
// B200 layout: the elementwise kernels are HBM streams, four elements per
// thread through 16-byte loads when every pointer is 16-byte aligned and
// the horizontal size is a multiple of 4 (scalar otherwise), grid-stride
// over a grid of a few waves; a thread walks the tracer blocks of its
// elements, so the shared operands are read once.  The vertical flux
// divergence marches one thread down each column for four tracers at once
// (consecutive threads = consecutive columns, so every level's loads
// coalesce), holding each tracer's three-layer window, gradients and
// previous interface flux in registers: every input is read once and every
// interface flux computed once (the reference's elementwise form
// recomputes each flux for both layers it bounds and re-reads the
// pressures for every tracer).
#include <algorithm>

#include "sht_common.cuh"

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

int grid_for(int64_t work, int threads) {
  int dev = 0, sms = 0;
  SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
  SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t per_wave = (int64_t)sms * (2048 / threads);
  return (int)std::max<int64_t>(1, std::min<int64_t>(div_up(work, threads), 4 * per_wave));
}

template <typename T> struct V4;
template <> struct V4<float> { using type = float4; };
template <> struct V4<double> { using type = double4; };

// ---------------------------------------------------- momentum/Bernoulli
template <typename T>
struct MomArgs {
  const T *zeta, *cor, *u, *v, *wu, *wv, *tv, *pg, *ge, *gn, *phi;
  T *mu, *mv, *bern;
  T rgas;
  int64_t n, horiz;
};

template <typename T>
__device__ __forceinline__ void momentum_point(const MomArgs<T>& a, T zeta, T cor, T u, T v,
                                               T wu, T wv, T tv, T pg, T ge, T gn, T phi, T& mu,
                                               T& mv, T& bern) {
  const T av = zeta + cor;
  const T pf = a.rgas * tv * pg;
  mu = av * v - wu - pf * ge;
  mv = -av * u - wv - pf * gn;
  bern = T(0.5) * (u * u + v * v) + phi;
}

template <typename T, bool VEC>
__global__ void __launch_bounds__(256) momentum_bernoulli_kernel(const MomArgs<T> a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if constexpr (VEC) {
    using V = typename V4<T>::type;
    const int64_t n4 = a.n / 4;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
      const int64_t e = 4 * q, h = e % a.horiz;
      const V z = __ldcs(reinterpret_cast<const V*>(a.zeta) + q);
      const V uu = __ldcs(reinterpret_cast<const V*>(a.u) + q);
      const V vv = __ldcs(reinterpret_cast<const V*>(a.v) + q);
      const V w1 = __ldcs(reinterpret_cast<const V*>(a.wu) + q);
      const V w2 = __ldcs(reinterpret_cast<const V*>(a.wv) + q);
      const V t = __ldcs(reinterpret_cast<const V*>(a.tv) + q);
      const V p = __ldcs(reinterpret_cast<const V*>(a.pg) + q);
      const V ph = __ldcs(reinterpret_cast<const V*>(a.phi) + q);
      const V c = __ldg(reinterpret_cast<const V*>(a.cor + h));
      const V ge = __ldg(reinterpret_cast<const V*>(a.ge + h));
      const V gn = __ldg(reinterpret_cast<const V*>(a.gn + h));
      V mu, mv, b;
      momentum_point(a, z.x, c.x, uu.x, vv.x, w1.x, w2.x, t.x, p.x, ge.x, gn.x, ph.x, mu.x, mv.x, b.x);
      momentum_point(a, z.y, c.y, uu.y, vv.y, w1.y, w2.y, t.y, p.y, ge.y, gn.y, ph.y, mu.y, mv.y, b.y);
      momentum_point(a, z.z, c.z, uu.z, vv.z, w1.z, w2.z, t.z, p.z, ge.z, gn.z, ph.z, mu.z, mv.z, b.z);
      momentum_point(a, z.w, c.w, uu.w, vv.w, w1.w, w2.w, t.w, p.w, ge.w, gn.w, ph.w, mu.w, mv.w, b.w);
      __stcs(reinterpret_cast<V*>(a.mu) + q, mu);
      __stcs(reinterpret_cast<V*>(a.mv) + q, mv);
      __stcs(reinterpret_cast<V*>(a.bern) + q, b);
    }
  } else {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.n; e += stride) {
      const int64_t h = e % a.horiz;
      momentum_point(a, a.zeta[e], a.cor[h], a.u[e], a.v[e], a.wu[e], a.wv[e], a.tv[e], a.pg[e],
                     a.ge[h], a.gn[h], a.phi[e], a.mu[e], a.mv[e], a.bern[e]);
    }
  }
}

// ------------------------------------------------ tracer flux / tendency
// A thread takes elements of the shared block and walks the tracer blocks,
// so dp, u, v (dp_t, dp) come from memory once, not once per tracer.
template <typename T>
struct FluxArgs {
  const T *dp, *s, *u, *v;  // dp, u, v: one block of `block` elements
  T *fx, *fy;
  int64_t blocks, block;
};

template <typename T, bool VEC>
__global__ void __launch_bounds__(256) tracer_flux_kernel(const FluxArgs<T> a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if constexpr (VEC) {
    using V = typename V4<T>::type;
    const int64_t nb4 = a.block / 4;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nb4; q += stride) {
      const V dp = __ldcs(reinterpret_cast<const V*>(a.dp) + q);
      const V u = __ldcs(reinterpret_cast<const V*>(a.u) + q);
      const V v = __ldcs(reinterpret_cast<const V*>(a.v) + q);
      for (int64_t b = 0; b < a.blocks; ++b) {
        const int64_t o = b * nb4 + q;
        const V s = __ldcs(reinterpret_cast<const V*>(a.s) + o);
        const V m = {dp.x * s.x, dp.y * s.y, dp.z * s.z, dp.w * s.w};
        __stcs(reinterpret_cast<V*>(a.fx) + o, V{m.x * u.x, m.y * u.y, m.z * u.z, m.w * u.w});
        __stcs(reinterpret_cast<V*>(a.fy) + o, V{m.x * v.x, m.y * v.y, m.z * v.z, m.w * v.w});
      }
    }
  } else {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.block; e += stride) {
      const T dp = a.dp[e], u = a.u[e], v = a.v[e];
      for (int64_t b = 0; b < a.blocks; ++b) {
        const int64_t o = b * a.block + e;
        const T m = dp * a.s[o];
        a.fx[o] = m * u;
        a.fy[o] = m * v;
      }
    }
  }
}

template <typename T>
struct TendArgs {
  const T *h, *vert, *s, *dpt, *dp;  // dpt, dp: one block
  T* out;
  int64_t blocks, block;
};

template <typename T>
__device__ __forceinline__ T tendency(T h, T vert, T s, T dpt, T dp) {
  return (-h - vert - s * dpt) / dp;
}

template <typename T, bool VEC>
__global__ void __launch_bounds__(256) scalar_tendency_kernel(const TendArgs<T> a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  if constexpr (VEC) {
    using V = typename V4<T>::type;
    const int64_t nb4 = a.block / 4;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nb4; q += stride) {
      const V dt = __ldcs(reinterpret_cast<const V*>(a.dpt) + q);
      const V dp = __ldcs(reinterpret_cast<const V*>(a.dp) + q);
      for (int64_t b = 0; b < a.blocks; ++b) {
        const int64_t o = b * nb4 + q;
        const V h = __ldcs(reinterpret_cast<const V*>(a.h) + o);
        const V vt = __ldcs(reinterpret_cast<const V*>(a.vert) + o);
        const V s = __ldcs(reinterpret_cast<const V*>(a.s) + o);
        __stcs(reinterpret_cast<V*>(a.out) + o,
               V{tendency(h.x, vt.x, s.x, dt.x, dp.x), tendency(h.y, vt.y, s.y, dt.y, dp.y),
                 tendency(h.z, vt.z, s.z, dt.z, dp.z), tendency(h.w, vt.w, s.w, dt.w, dp.w)});
      }
    }
  } else {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.block; e += stride) {
      const T dt = a.dpt[e], dp = a.dp[e];
      for (int64_t b = 0; b < a.blocks; ++b) {
        const int64_t o = b * a.block + e;
        a.out[o] = tendency(a.h[o], a.vert[o], a.s[o], dt, dp);
      }
    }
  }
}

// ------------------------------------------- vertical flux divergence
template <typename T>
struct VfdArgs {
  const T *s, *w, *pf, *ph;  // s: [B][nlev][horiz]; w, ph: [nlev+1][horiz]; pf: [nlev][horiz]
  T* out;                    // [B][nlev][horiz]
  int nlev, b0;              // tracer blocks b0 .. b0 + NT - 1 in this launch
  int64_t horiz;
};

// Van Leer gradient of layer k from its window (s, p at k-1, k, k+1); the
// boundary layers take the one-sided gradient to their one neighbour.
template <typename T>
__device__ __forceinline__ T layer_gradient(int k, int nlev, T sm, T s0, T sp, T pm, T p0, T pp) {
  if (k > 0 && k + 1 < nlev) {
    const T ga = (s0 - sm) / (p0 - pm);
    const T gb = (sp - s0) / (pp - p0);
    const T prod = ga * gb;
    return prod > T(0) ? T(2) * prod / (ga + gb) : T(0);
  }
  if (k == 0) return (sp - s0) / (pp - p0);
  return (s0 - sm) / (p0 - pm);
}

// Flux through interface j (0 < j < nlev) from the two layers around it:
// upstream layer j-1 (value sa, gradient ga, pressure pa) when w >= 0, else
// layer j (sb, gb, pb); the face value is bounded by the two layers.
template <typename T>
__device__ __forceinline__ T interface_flux(T wj, T phj, T sa, T ga, T pa, T sb, T gb, T pb) {
  const bool from_above = wj >= T(0);
  const T su = from_above ? sa : sb;
  const T gu = from_above ? ga : gb;
  const T pu = from_above ? pa : pb;
  T face = su + gu * (phj - pu);
  const T lo = sa < sb ? sa : sb, hi = sa > sb ? sa : sb;
  face = face > lo ? face : lo;
  face = face < hi ? face : hi;
  return wj * face;
}

// One thread marches one column down the levels for NT tracers at once:
// the pressures and the interface velocity of a level are loaded once for
// all of them, and the NT recurrences are independent work between loads.
// (Without the one-level prefetch: 2.40 ms at T511 L40 x 8 tracers, against
// 1.16 with it; splitting a column into chunks marched by separate threads,
// each forming its top interface's flux from the four layers around it,
// measured 2.81.)
template <typename T, int NT>
__global__ void __launch_bounds__(256) vertical_flux_divergence_kernel(const VfdArgs<T> a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int nlev = a.nlev;
  const int64_t H = a.horiz;
  for (int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; col < H; col += stride) {
    const T* s[NT];
    T* out[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      s[t] = a.s + (int64_t)(a.b0 + t) * nlev * H + col;
      out[t] = a.out + (int64_t)(a.b0 + t) * nlev * H + col;
    }
    const T* pf = a.pf + col;
    const T* w = a.w + col;
    const T* ph = a.ph + col;
    T s0[NT], sp[NT], g0[NT], fa[NT], s_pre[NT];
    T p_0 = __ldg(pf), p_p = nlev > 1 ? __ldg(pf + H) : T(0);
    // One level of loads in flight ahead of the arithmetic: the values of
    // level k + 2 (interface k + 1) are loaded during iteration k - 1.
    T p_pre = nlev > 2 ? __ldg(pf + 2 * H) : T(0);
    T w_pre = nlev > 1 ? __ldg(w + H) : T(0);
    T ph_pre = nlev > 1 ? __ldg(ph + H) : T(0);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      s0[t] = __ldcs(s[t]);
      sp[t] = nlev > 1 ? __ldcs(s[t] + H) : T(0);
      s_pre[t] = nlev > 2 ? __ldcs(s[t] + 2 * H) : T(0);
      g0[t] = nlev > 1 ? layer_gradient(0, nlev, T(0), s0[t], sp[t], T(0), p_0, p_p) : T(0);
      fa[t] = T(0);  // no flux through the top
    }
    for (int k = 0; k < nlev; ++k) {
      const bool inner = k + 1 < nlev;
      const T p_next = p_pre, wj = w_pre, phj = ph_pre;
      T s_next[NT];
#pragma unroll
      for (int t = 0; t < NT; ++t) s_next[t] = s_pre[t];
      // prefetch level k + 3 and interface k + 2
      p_pre = k + 3 < nlev ? __ldg(pf + (int64_t)(k + 3) * H) : T(0);
      w_pre = k + 2 < nlev ? __ldg(w + (int64_t)(k + 2) * H) : T(0);
      ph_pre = k + 2 < nlev ? __ldg(ph + (int64_t)(k + 2) * H) : T(0);
#pragma unroll
      for (int t = 0; t < NT; ++t)
        s_pre[t] = k + 3 < nlev ? __ldcs(s[t] + (int64_t)(k + 3) * H) : T(0);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        T fb = T(0), g_next = T(0);
        if (inner) {
          g_next = layer_gradient(k + 1, nlev, s0[t], sp[t], s_next[t], p_0, p_p, p_next);
          fb = interface_flux(wj, phj, s0[t], g0[t], p_0, sp[t], g_next, p_p);
        }
        __stcs(out[t] + (int64_t)k * H, fb - fa[t]);
        fa[t] = fb;
        s0[t] = sp[t];
        sp[t] = s_next[t];
        g0[t] = g_next;
      }
      p_0 = p_p;
      p_p = p_next;
    }
  }
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

template <typename T>
bool vec_ok(int64_t n, int64_t period, std::initializer_list<const void*> ptrs) {
  if (sizeof(T) != 4 || n % 4 != 0 || period % 4 != 0) return false;
  for (const void* p : ptrs)
    if (!aligned16(p)) return false;
  return true;
}

void require(std::initializer_list<const void*> ptrs) {
  for (const void* p : ptrs) SHT_REQUIRE(p != nullptr, "null array pointer");
}

}  // namespace
}  // namespace sht

using namespace sht;

extern "C" {

int sht_rhs_momentum_bernoulli(int precision, int64_t nlev, int64_t horiz, const void* zeta,
                               const void* coriolis, const void* u, const void* v, const void* wu,
                               const void* wv, const void* tv, const void* pg,
                               const void* grad_lnps_east, const void* grad_lnps_north,
                               const void* geopotential, double gas_constant, void* mu, void* mv,
                               void* bernoulli, void* stream) {
  return guarded([&] {
    require({zeta, coriolis, u, v, wu, wv, tv, pg, grad_lnps_east, grad_lnps_north, geopotential,
             mu, mv, bernoulli});
    SHT_REQUIRE(nlev >= 1 && horiz >= 1, "nlev and horiz must be positive");
    SHT_REQUIRE(precision == SHT_PREC_F64 || precision == SHT_PREC_F32,
                "the RHS kernels run in float32 or float64");
    const int64_t n = nlev * horiz;
    cudaStream_t s = (cudaStream_t)stream;
    auto go = [&](auto tag) {
      using T = decltype(tag);
      MomArgs<T> a{(const T*)zeta, (const T*)coriolis, (const T*)u, (const T*)v, (const T*)wu,
                   (const T*)wv, (const T*)tv, (const T*)pg, (const T*)grad_lnps_east,
                   (const T*)grad_lnps_north, (const T*)geopotential, (T*)mu, (T*)mv,
                   (T*)bernoulli, (T)gas_constant, n, horiz};
      if constexpr (sizeof(T) == 4) {  // 16-byte vectors: float4
        if (vec_ok<T>(n, horiz, {zeta, coriolis, u, v, wu, wv, tv, pg, grad_lnps_east,
                               grad_lnps_north, geopotential, mu, mv, bernoulli})) {
          momentum_bernoulli_kernel<T, true><<<grid_for(n / 4, 256), 256, 0, s>>>(a);
          return;
        }
      }
      momentum_bernoulli_kernel<T, false><<<grid_for(n, 256), 256, 0, s>>>(a);
    };
    if (precision == SHT_PREC_F64) go(double{}); else go(float{});
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

int sht_rhs_tracer_flux(int precision, int64_t blocks, int64_t nlev, int64_t horiz,
                        const void* dp, const void* scalar, const void* u, const void* v,
                        void* flux_east, void* flux_north, void* stream) {
  return guarded([&] {
    require({dp, scalar, u, v, flux_east, flux_north});
    SHT_REQUIRE(blocks >= 1 && nlev >= 1 && horiz >= 1, "sizes must be positive");
    SHT_REQUIRE(precision == SHT_PREC_F64 || precision == SHT_PREC_F32,
                "the RHS kernels run in float32 or float64");
    const int64_t block = nlev * horiz, n = blocks * block;
    cudaStream_t s = (cudaStream_t)stream;
    auto go = [&](auto tag) {
      using T = decltype(tag);
      FluxArgs<T> a{(const T*)dp, (const T*)scalar, (const T*)u, (const T*)v, (T*)flux_east,
                    (T*)flux_north, blocks, block};
      if constexpr (sizeof(T) == 4) {  // 16-byte vectors: float4
        if (vec_ok<T>(n, block, {dp, scalar, u, v, flux_east, flux_north})) {
          tracer_flux_kernel<T, true><<<grid_for(block / 4, 256), 256, 0, s>>>(a);
          return;
        }
      }
      tracer_flux_kernel<T, false><<<grid_for(block, 256), 256, 0, s>>>(a);
    };
    if (precision == SHT_PREC_F64) go(double{}); else go(float{});
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

int sht_rhs_scalar_tendency(int precision, int64_t blocks, int64_t nlev, int64_t horiz,
                            const void* horizontal, const void* vertical, const void* scalar,
                            const void* dp_t, const void* dp, void* out, void* stream) {
  return guarded([&] {
    require({horizontal, vertical, scalar, dp_t, dp, out});
    SHT_REQUIRE(blocks >= 1 && nlev >= 1 && horiz >= 1, "sizes must be positive");
    SHT_REQUIRE(precision == SHT_PREC_F64 || precision == SHT_PREC_F32,
                "the RHS kernels run in float32 or float64");
    const int64_t block = nlev * horiz, n = blocks * block;
    cudaStream_t s = (cudaStream_t)stream;
    auto go = [&](auto tag) {
      using T = decltype(tag);
      TendArgs<T> a{(const T*)horizontal, (const T*)vertical, (const T*)scalar, (const T*)dp_t,
                    (const T*)dp, (T*)out, blocks, block};
      if constexpr (sizeof(T) == 4) {  // 16-byte vectors: float4
        if (vec_ok<T>(n, block, {horizontal, vertical, scalar, dp_t, dp, out})) {
          scalar_tendency_kernel<T, true><<<grid_for(block / 4, 256), 256, 0, s>>>(a);
          return;
        }
      }
      scalar_tendency_kernel<T, false><<<grid_for(block, 256), 256, 0, s>>>(a);
    };
    if (precision == SHT_PREC_F64) go(double{}); else go(float{});
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

int sht_rhs_vertical_flux_divergence(int precision, int64_t blocks, int64_t nlev, int64_t horiz,
                                     const void* scalar, const void* omega_half,
                                     const void* p_full, const void* p_half, void* out,
                                     void* stream) {
  return guarded([&] {
    require({scalar, omega_half, p_full, p_half, out});
    SHT_REQUIRE(blocks >= 1 && nlev >= 1 && horiz >= 1, "sizes must be positive");
    SHT_REQUIRE(nlev < (1 << 20), "nlev too large");
    SHT_REQUIRE(precision == SHT_PREC_F64 || precision == SHT_PREC_F32,
                "the RHS kernels run in float32 or float64");
    SHT_REQUIRE(blocks < (1 << 30), "too many tracer blocks");
    cudaStream_t s = (cudaStream_t)stream;
    auto go = [&](auto tag) {
      using T = decltype(tag);
      VfdArgs<T> a{(const T*)scalar, (const T*)omega_half, (const T*)p_full, (const T*)p_half,
                   (T*)out, (int)nlev, 0, horiz};
      const int grid = grid_for(horiz, 256);
      // four tracers per thread, then the rest one at a time
      for (; a.b0 + 4 <= blocks; a.b0 += 4)
        vertical_flux_divergence_kernel<T, 4><<<grid, 256, 0, s>>>(a);
      for (; a.b0 < blocks; ++a.b0) vertical_flux_divergence_kernel<T, 1><<<grid, 256, 0, s>>>(a);
    };
    if (precision == SHT_PREC_F64) go(double{}); else go(float{});
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

}  // extern "C"
