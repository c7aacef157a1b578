// Spectral fields evaluated at arbitrary points: the reference's
// spectral/sampling.py sample_scalar / sample_gradient (host path
// sampling.py:382-478: per point the orthonormal P_n^m(sin phi) and
// dP/dphi of legendre.py, amplitudes sum_n c_nm P_nm, then
// sum_m (m ? 2 : 1) Re(A_m e^{i m lambda})).
//
// B200 layout: a CTA takes 32 points, one per lane, and its 12 warps split
// the orders into contiguous bands of equal triangular cost.  Every lane of
// a warp walks the same (m, n) sequence for its own point, so each
// coefficient and recurrence factor is one broadcast load for the 32
// points (a CTA per point re-read the whole spectrum per point, ~8 MB at
// T511, and ran at ~3 % of the FP64 rate).  A warp carries the sectoral
// value P_mm from the first order of its band by the reference's product
// (the same multiplications in the same order, from m = 1), runs the n
// recurrence with the x-independent factors tabulated once per truncation
// ([m][n]), applies the phase and adds up to 4 fields per pass; the bands'
// partial sums are added in band order.  FP64 throughout, the products and
// sums unfused (__dmul_rn / __dadd_rn) as the reference's numpy evaluates
// them, so each P value is the reference's rounding.
#include <cmath>
#include <vector>

#include "sht_common.cuh"

struct sht_sampler {
  int T = 0, device = 0;
  double* d_a = nullptr;   // [m][n] recurrence factor sqrt((4n^2-1)/(n^2-m^2))
  double* d_b = nullptr;   // [m][n] sqrt(((n-1)^2-m^2)/(4(n-1)^2-1))
  double* d_c = nullptr;   // [m][n] derivative factor sqrt((n^2-m^2)(2n+1)/(2n-1))
  double* d_s = nullptr;   // [m] sqrt((2m+1)/(2m)) of the sectoral step
  int* d_band = nullptr;   // [kSampleWarps + 1] first order of each warp's band
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

constexpr int kSamplePoints = 32;  // points per CTA, one per lane
constexpr int kSampleWarps = 12;   // order bands per CTA, one per warp
constexpr int kMaxFieldsPerPass = 4;

struct SampleArgs {
  int T, F, f0;                 // truncation; fields; first field of this pass
  int64_t npoints;
  const double2* coeff;         // [F][m][n] complex, n fastest
  const double *lat, *lon;      // radians
  const double *a, *b, *c, *s;  // tables
  double radius;
  double *out0, *out1;          // [F][npoints]: scalar, or east / north
};

template <int NF, bool GRAD>
__global__ void __launch_bounds__(kSamplePoints * kSampleWarps) sample_kernel(const SampleArgs g,
                                                                        const int* __restrict__ band) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t p = (int64_t)blockIdx.x * kSamplePoints + lane;
  const bool live = p < g.npoints;  // dead lanes follow along on a dummy point
  const int T = g.T, T1 = T + 1;
  const double lat = live ? g.lat[p] : 0.0, lon = live ? g.lon[p] : 0.0;
  const double x = sin(lat);
  const double root = __dsqrt_rn(fmax(0.0, __dsub_rn(1.0, __dmul_rn(x, x))));
  const double denom = __dsub_rn(__dmul_rn(x, x), 1.0);
  double acc0[NF], acc1[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) acc0[f] = acc1[f] = 0.0;
  const int m0 = band[warp], m1 = band[warp + 1];
  // sectoral value P_mm at the band's first order, by the product from m = 1
  double diag = 1.0 / sqrt(4.0 * kPi);
  for (int k = 1; k <= m0; ++k) diag = __dmul_rn(__dmul_rn(-g.s[k], root), diag);
  for (int m = m0; m < m1; ++m) {
    if (m > m0) diag = __dmul_rn(__dmul_rn(-g.s[m], root), diag);
    const double* arow = g.a + (int64_t)m * T1;
    const double* brow = g.b + (int64_t)m * T1;
    const double* crow = g.c + (int64_t)m * T1;
    double A[NF][2], D[NF][2];
    const double2* cf[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      cf[f] = g.coeff + ((int64_t)(g.f0 + f) * T1 + m) * T1;
      const double2 v = cf[f][m];
      A[f][0] = __dmul_rn(v.x, diag);
      A[f][1] = __dmul_rn(v.y, diag);
      D[f][0] = D[f][1] = 0.0;
    }
    if (GRAD && m >= 1) {
      const double d = __ddiv_rn(__dmul_rn(root, __dmul_rn(__dmul_rn((double)m, x), diag)), denom);
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double2 v = cf[f][m];
        D[f][0] = __dmul_rn(v.x, d);
        D[f][1] = __dmul_rn(v.y, d);
      }
    }
    double p2 = 0.0, p1 = diag;
    for (int n = m + 1; n <= T; ++n) {
      const double pn = n == m + 1
                            ? __dmul_rn(__dmul_rn(__dsqrt_rn((double)(2 * m + 3)), x), diag)
                            : __dmul_rn(arow[n], __dsub_rn(__dmul_rn(x, p1), __dmul_rn(brow[n], p2)));
      double dn = 0.0;
      if (GRAD) {
        const double num = __dsub_rn(__dmul_rn(__dmul_rn((double)n, x), pn), __dmul_rn(crow[n], p1));
        dn = __ddiv_rn(__dmul_rn(root, num), denom);
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double2 v = cf[f][n];
        A[f][0] = __dadd_rn(A[f][0], __dmul_rn(v.x, pn));
        A[f][1] = __dadd_rn(A[f][1], __dmul_rn(v.y, pn));
        if (GRAD) {
          D[f][0] = __dadd_rn(D[f][0], __dmul_rn(v.x, dn));
          D[f][1] = __dadd_rn(D[f][1], __dmul_rn(v.y, dn));
        }
      }
      p2 = p1;
      p1 = pn;
    }
    double sn, cs;
    sincos((double)m * lon, &sn, &cs);
    const double mult = m == 0 ? 1.0 : 2.0;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      // Re(A e^{i m lon}) and, for the gradient, Re(i m A e^{i m lon}), Re(D e^{i m lon})
      const double re = __dsub_rn(__dmul_rn(A[f][0], cs), __dmul_rn(A[f][1], sn));
      const double im = __dadd_rn(__dmul_rn(A[f][0], sn), __dmul_rn(A[f][1], cs));
      if (GRAD) {
        acc0[f] = __dadd_rn(acc0[f], __dmul_rn(mult, __dmul_rn(-(double)m, im)));
        acc1[f] = __dadd_rn(acc1[f], __dmul_rn(mult, __dsub_rn(__dmul_rn(D[f][0], cs),
                                                                __dmul_rn(D[f][1], sn))));
      } else {
        acc0[f] = __dadd_rn(acc0[f], __dmul_rn(mult, re));
      }
    }
  }
  // the bands' partial sums, added in band order
  __shared__ double red[kSampleWarps][2][NF][kSamplePoints];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    red[warp][0][f][lane] = acc0[f];
    red[warp][1][f][lane] = acc1[f];
  }
  __syncthreads();
  if (warp < NF) {
    const int f = warp;
    double s0 = red[0][0][f][lane], s1 = red[0][1][f][lane];
    for (int w = 1; w < kSampleWarps; ++w) {
      s0 += red[w][0][f][lane];
      s1 += red[w][1][f][lane];
    }
    if (live) {
      const int64_t o = (int64_t)(g.f0 + f) * g.npoints + p;
      if (GRAD) {
        g.out0[o] = s0 / (g.radius * cos(lat));
        g.out1[o] = s1 / g.radius;
      } else {
        g.out0[o] = s0;
      }
    }
  }
}

// The packed real basis blocks the reference's device sampler contracts
// (spectral/sampling.py:198-237): one thread per (order m, point p), the
// point fastest.  For the packed (n, m) row k (orders below m fill
// T + 1 - m' rows each, n fastest) the scalar block holds
// mult P cos(m lam) in row k and -mult P sin(m lam) in row K + k; the
// gradient blocks hold -m mult P sin / -m mult P cos (zonal) and
// mult dP cos / -mult dP sin (meridional), mult = 1 at m = 0 and 2 above.
// The P and dP values are the sampler's recurrence, unfused.
struct BasisArgs {
  int T;
  int64_t npoints, ktri;
  const double *lat, *lon;
  const double *a, *b, *c, *s;
  void *out0, *out1;  // [2 K][npoints] of OUT
};

template <typename OUT, bool GRAD>
__global__ void __launch_bounds__(256) packed_basis_kernel(const BasisArgs g) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)(g.T + 1) * g.npoints) return;
  const int64_t p = i % g.npoints;
  const int m = (int)(i / g.npoints);
  const int T = g.T, T1 = T + 1;
  const double x = sin(g.lat[p]);
  const double root = __dsqrt_rn(fmax(0.0, __dsub_rn(1.0, __dmul_rn(x, x))));
  const double denom = __dsub_rn(__dmul_rn(x, x), 1.0);
  double diag = 1.0 / sqrt(4.0 * kPi);
  for (int k = 1; k <= m; ++k) diag = __dmul_rn(__dmul_rn(-g.s[k], root), diag);
  double sn, cs;
  sincos((double)m * g.lon[p], &sn, &cs);
  const double mult = m == 0 ? 1.0 : 2.0;
  const double mm = mult * (double)m;
  OUT* b0 = static_cast<OUT*>(g.out0);
  OUT* b1 = static_cast<OUT*>(g.out1);
  const int64_t np = g.npoints, kk = g.ktri;
  auto emit = [&](int64_t k, double P, double dP) {
    if (GRAD) {
      b0[k * np + p] = (OUT)(-__dmul_rn(__dmul_rn(mm, P), sn));
      b0[(k + kk) * np + p] = (OUT)(-__dmul_rn(__dmul_rn(mm, P), cs));
      b1[k * np + p] = (OUT)__dmul_rn(__dmul_rn(mult, dP), cs);
      b1[(k + kk) * np + p] = (OUT)(-__dmul_rn(__dmul_rn(mult, dP), sn));
    } else {
      b0[k * np + p] = (OUT)__dmul_rn(__dmul_rn(mult, P), cs);
      b0[(k + kk) * np + p] = (OUT)(-__dmul_rn(__dmul_rn(mult, P), sn));
    }
  };
  int64_t k = (int64_t)m * T1 - (int64_t)m * (m - 1) / 2;
  const double d0 =
      m >= 1 ? __ddiv_rn(__dmul_rn(root, __dmul_rn(__dmul_rn((double)m, x), diag)), denom) : 0.0;
  emit(k++, diag, d0);
  const double* arow = g.a + (int64_t)m * T1;
  const double* brow = g.b + (int64_t)m * T1;
  const double* crow = g.c + (int64_t)m * T1;
  double p2 = 0.0, p1 = diag;
  for (int n = m + 1; n <= T; ++n) {
    const double pn = n == m + 1
                          ? __dmul_rn(__dmul_rn(__dsqrt_rn((double)(2 * m + 3)), x), diag)
                          : __dmul_rn(arow[n], __dsub_rn(__dmul_rn(x, p1), __dmul_rn(brow[n], p2)));
    const double num = __dsub_rn(__dmul_rn(__dmul_rn((double)n, x), pn), __dmul_rn(crow[n], p1));
    emit(k++, pn, __ddiv_rn(__dmul_rn(root, num), denom));
    p2 = p1;
    p1 = pn;
  }
}

template <bool GRAD>
void launch_passes(SampleArgs g, const int* band, cudaStream_t s) {
  const unsigned blocks = (unsigned)div_up(g.npoints, kSamplePoints);
  const int threads = kSamplePoints * kSampleWarps;
  for (g.f0 = 0; g.f0 < g.F;) {
    const int left = g.F - g.f0;
    if (left >= 4) {
      sample_kernel<4, GRAD><<<blocks, threads, 0, s>>>(g, band);
      g.f0 += 4;
    } else if (left >= 2) {
      sample_kernel<2, GRAD><<<blocks, threads, 0, s>>>(g, band);
      g.f0 += 2;
    } else {
      sample_kernel<1, GRAD><<<blocks, threads, 0, s>>>(g, band);
      g.f0 += 1;
    }
    SHT_CUDA_OR_THROW(cudaGetLastError());
  }
}

// Order bands of equal cost: order m costs its T + 1 - m recurrence terms
// plus a fixed share for its sectoral step, phase and set-up.
std::vector<int> order_bands(int T) {
  const int T1 = T + 1;
  auto cost = [&](int m) { return (double)(T1 - m) + 24.0; };
  double total = 0.0;
  for (int m = 0; m <= T; ++m) total += cost(m);
  std::vector<int> band(kSampleWarps + 1, T1);
  band[0] = 0;
  double run = 0.0;
  int w = 1;
  for (int m = 0; m <= T && w < kSampleWarps; ++m) {
    run += cost(m);
    while (w < kSampleWarps && run >= total * w / kSampleWarps) band[w++] = m + 1;
  }
  return band;
}

}  // namespace
}  // namespace sht

using namespace sht;

extern "C" {

int sht_sampler_create(int truncation, sht_sampler** out) {
  return guarded([&] {
    SHT_REQUIRE(out != nullptr, "null output handle");
    *out = nullptr;
    SHT_REQUIRE(truncation >= 0 && truncation <= 4096, "truncation must be in [0, 4096]");
    const int T = truncation, T1 = T + 1;
    std::vector<double> a((size_t)T1 * T1, 0.0), b((size_t)T1 * T1, 0.0), c((size_t)T1 * T1, 0.0),
        sv(T1, 0.0);
    // The factors of the orthonormal recurrence, formed as the plan's
    // Legendre tables form them (no fused operations).
    for (int m = 0; m <= T; ++m)
      for (int n = m + 1; n <= T; ++n) {
        const double nn = n, mm = m, n1 = nn - 1.0;
        const double nm2 = (double)((long long)n * n - (long long)m * m);
        a[(size_t)m * T1 + n] = std::sqrt((4.0 * nn * nn - 1.0) / nm2);
        b[(size_t)m * T1 + n] = std::sqrt((n1 * n1 - mm * mm) / (4.0 * n1 * n1 - 1.0));
        c[(size_t)m * T1 + n] = std::sqrt(nm2 * (2.0 * nn + 1.0) / (2.0 * nn - 1.0));
      }
    for (int k = 1; k <= T; ++k) sv[k] = std::sqrt((double)(2 * k + 1) / (2.0 * k));
    auto* h = new sht_sampler;
    try {
      h->T = T;
      SHT_CUDA_OR_THROW(cudaGetDevice(&h->device));
      for (double** d : {&h->d_a, &h->d_b, &h->d_c})
        SHT_CUDA_OR_THROW(cudaMalloc(d, a.size() * sizeof(double)));
      SHT_CUDA_OR_THROW(cudaMalloc(&h->d_s, sv.size() * sizeof(double)));
      const std::vector<int> band = order_bands(T);
      SHT_CUDA_OR_THROW(cudaMalloc(&h->d_band, band.size() * sizeof(int)));
      upload_now(h->d_band, band.data(), band.size() * sizeof(int));
      upload_now(h->d_a, a.data(), a.size() * sizeof(double));
      upload_now(h->d_b, b.data(), b.size() * sizeof(double));
      upload_now(h->d_c, c.data(), c.size() * sizeof(double));
      upload_now(h->d_s, sv.data(), sv.size() * sizeof(double));
    } catch (...) {
      cudaFree(h->d_a);
      cudaFree(h->d_b);
      cudaFree(h->d_c);
      cudaFree(h->d_s);
      cudaFree(h->d_band);
      delete h;
      throw;
    }
    *out = h;
  });
}

int sht_sampler_destroy(sht_sampler* h) {
  return guarded([&] {
    if (!h) return;
    cudaFree(h->d_a);
    cudaFree(h->d_b);
    cudaFree(h->d_c);
    cudaFree(h->d_s);
    cudaFree(h->d_band);
    delete h;
  });
}

int sht_sample(sht_sampler* h, const void* coeff_mn, int64_t fields, int64_t npoints,
               const double* lat_rad, const double* lon_rad, int gradient, double radius,
               double* out0, double* out1, void* stream) {
  return guarded([&] {
    SHT_REQUIRE(h != nullptr, "null sampler");
    SHT_REQUIRE(coeff_mn && lat_rad && lon_rad && out0, "null array pointer");
    SHT_REQUIRE(fields >= 1 && fields < (1 << 24), "fields must be in [1, 2^24)");
    SHT_REQUIRE(npoints >= 1 && npoints < (1LL << 31), "npoints must be in [1, 2^31)");
    if (gradient) {
      SHT_REQUIRE(out1 != nullptr, "null northward output");
      SHT_REQUIRE(std::isfinite(radius) && radius > 0.0, "radius must be finite and positive");
    }
    int dev = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
    SHT_REQUIRE(dev == h->device, "the sampler lives on another device");
    SampleArgs g{h->T, (int)fields, 0, npoints, (const double2*)coeff_mn, lat_rad, lon_rad,
                 h->d_a, h->d_b, h->d_c, h->d_s, radius, out0, out1};
    cudaStream_t s = (cudaStream_t)stream;
    if (gradient) launch_passes<true>(g, h->d_band, s);
    else launch_passes<false>(g, h->d_band, s);
  });
}

int sht_sample_packed_basis(sht_sampler* h, int64_t npoints, const double* lat_rad,
                            const double* lon_rad, int gradient, int out_precision, void* out0,
                            void* out1, void* stream) {
  return guarded([&] {
    SHT_REQUIRE(h != nullptr, "null sampler");
    SHT_REQUIRE(lat_rad && lon_rad && out0, "null array pointer");
    SHT_REQUIRE(!gradient || out1 != nullptr, "null meridional block");
    SHT_REQUIRE(npoints >= 1 && npoints < (1LL << 31), "npoints must be in [1, 2^31)");
    SHT_REQUIRE(out_precision == SHT_PREC_F64 || out_precision == SHT_PREC_F32,
                "out_precision must be SHT_PREC_F64 or SHT_PREC_F32");
    int dev = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
    SHT_REQUIRE(dev == h->device, "the sampler lives on another device");
    const int64_t ktri = (int64_t)(h->T + 1) * (h->T + 2) / 2;
    BasisArgs g{h->T, npoints, ktri, lat_rad, lon_rad, h->d_a, h->d_b, h->d_c, h->d_s, out0,
                out1};
    const int64_t threads = (int64_t)(h->T + 1) * npoints;
    const unsigned blocks = (unsigned)div_up(threads, 256);
    cudaStream_t s = (cudaStream_t)stream;
    if (out_precision == SHT_PREC_F64) {
      if (gradient) packed_basis_kernel<double, true><<<blocks, 256, 0, s>>>(g);
      else packed_basis_kernel<double, false><<<blocks, 256, 0, s>>>(g);
    } else {
      if (gradient) packed_basis_kernel<float, true><<<blocks, 256, 0, s>>>(g);
      else packed_basis_kernel<float, false><<<blocks, 256, 0, s>>>(g);
    }
    SHT_CUDA_OR_THROW(cudaGetLastError());
  });
}

}  // extern "C"
