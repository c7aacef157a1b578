// Longitude real FFTs that write and read the equator-folded Fourier waist.
//
// Forward (grid -> waist): rows of nlon reals are transformed as complex
// sequences of L = nlon/2 (z_k = x_2k + i x_2k+1) by a shared-memory Stockham
// FFT, untangled into the real-input spectrum X_m, scaled by 1/nlon and cut
// to m <= T (the reference's rfft(f)/nlon[..., :T+1], transform.py:1386-1390),
// then folded across the equator: S = X(row h) + X(mirror row), D = X(h) -
// X(mirror).  The waist layout is [m][s][h][r] with the row index r = 2*plane
// + (re, im) innermost, which is the operand layout of the per-order Legendre
// contraction, so no separate transpose kernel exists.
//
// Inverse (waist -> grid): the folded synthesis output is unfolded (X(h) = S
// + D, X(mirror) = S - D), optionally combined (zonal i*m factor, gradient
// metric factors, the (u, v) combination of the vector synthesis), entangled
// into a length-L complex sequence and inverted; the result equals
// irfft(nlon * W) of the reference (transform.py:1654-1702), which discards
// Imag(W_0) and has no Nyquist term because T < nlon/2.
#include "sht_plan.h"

namespace sht {
namespace {

template <typename T> using V2 = typename Vec2<T>::type;

template <typename T>
__device__ __forceinline__ V2<T> cmul(V2<T> a, V2<T> b) {
  return mk2<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ V2<T> cadd(V2<T> a, V2<T> b) { return mk2<T>(a.x + b.x, a.y + b.y); }
template <typename T>
__device__ __forceinline__ V2<T> csub(V2<T> a, V2<T> b) { return mk2<T>(a.x - b.x, a.y - b.y); }
template <typename T>
__device__ __forceinline__ V2<T> cconj(V2<T> a) { return mk2<T>(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <typename T>
__device__ __forceinline__ V2<T> rot90(V2<T> a, bool inv) {
  return inv ? mk2<T>(-a.y, a.x) : mk2<T>(a.y, -a.x);
}

// In-register DFTs of small radix.  Forward uses exp(-2 pi i rs/R).
template <typename T>
__device__ __forceinline__ void dft2(V2<T>* v) {
  V2<T> a = v[0], b = v[1];
  v[0] = cadd<T>(a, b);
  v[1] = csub<T>(a, b);
}
template <typename T>
__device__ __forceinline__ void dft3(V2<T>* v, bool inv) {
  const T c1 = T(-0.5);
  const T s1 = inv ? T(0.86602540378443864676) : T(-0.86602540378443864676);
  V2<T> a = v[0], b = v[1], c = v[2];
  V2<T> t1 = cadd<T>(b, c), t2 = csub<T>(b, c);
  v[0] = cadd<T>(a, t1);
  V2<T> m1 = mk2<T>(a.x + c1 * t1.x, a.y + c1 * t1.y);
  V2<T> m2 = mk2<T>(-s1 * t2.y, s1 * t2.x);  // i * s1 * t2
  v[1] = cadd<T>(m1, m2);
  v[2] = csub<T>(m1, m2);
}
template <typename T>
__device__ __forceinline__ void dft4(V2<T>* v, bool inv) {
  V2<T> a0 = cadd<T>(v[0], v[2]), a1 = csub<T>(v[0], v[2]);
  V2<T> b0 = cadd<T>(v[1], v[3]), b1 = rot90<T>(csub<T>(v[1], v[3]), inv);
  v[0] = cadd<T>(a0, b0);
  v[2] = csub<T>(a0, b0);
  v[1] = cadd<T>(a1, b1);
  v[3] = csub<T>(a1, b1);
}
template <typename T>
__device__ __forceinline__ void dft5(V2<T>* v, bool inv) {
  const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);
  const T s1 = inv ? T(0.95105651629515357212) : T(-0.95105651629515357212);
  const T s2 = inv ? T(0.58778525229247312917) : T(-0.58778525229247312917);
  V2<T> a = v[0];
  V2<T> t1 = cadd<T>(v[1], v[4]), t2 = csub<T>(v[1], v[4]);
  V2<T> t3 = cadd<T>(v[2], v[3]), t4 = csub<T>(v[2], v[3]);
  v[0] = mk2<T>(a.x + t1.x + t3.x, a.y + t1.y + t3.y);
  V2<T> r1 = mk2<T>(a.x + c1 * t1.x + c2 * t3.x, a.y + c1 * t1.y + c2 * t3.y);
  V2<T> r2 = mk2<T>(a.x + c2 * t1.x + c1 * t3.x, a.y + c2 * t1.y + c1 * t3.y);
  // i*(s1 t2 + s2 t4) and i*(s2 t2 - s1 t4)
  V2<T> i1 = mk2<T>(-(s1 * t2.y + s2 * t4.y), s1 * t2.x + s2 * t4.x);
  V2<T> i2 = mk2<T>(-(s2 * t2.y - s1 * t4.y), s2 * t2.x - s1 * t4.x);
  v[1] = cadd<T>(r1, i1);
  v[4] = csub<T>(r1, i1);
  v[2] = cadd<T>(r2, i2);
  v[3] = csub<T>(r2, i2);
}
template <typename T>
__device__ __forceinline__ void dft8(V2<T>* v, bool inv) {
  // radix-2 x 4: even/odd halves then combine with exp(-2 pi i k/8).
  V2<T> e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  dft4<T>(e, inv);
  dft4<T>(o, inv);
  const T r = T(0.70710678118654752440);
  // w^1 = (r, -r) forward, (r, r) inverse; w^2 = -i / +i; w^3 = (-r, -r) / (-r, r)
  o[1] = cmul<T>(o[1], mk2<T>(r, inv ? r : -r));
  o[2] = rot90<T>(o[2], inv);
  o[3] = cmul<T>(o[3], mk2<T>(-r, inv ? r : -r));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd<T>(e[k], o[k]);
    v[k + 4] = csub<T>(e[k], o[k]);
  }
}
template <typename T>
__device__ __forceinline__ void dft16(V2<T>* v, const V2<T>* w16, bool inv) {
  // 4 x 4: columns, twiddle, rows.  w16[k] = exp(-2 pi i k / 16).
  V2<T> a[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j) a[i][j] = v[j * 4 + i];
    dft4<T>(a[i], inv);
  }
#pragma unroll
  for (int i = 1; i < 4; ++i)
#pragma unroll
    for (int j = 1; j < 4; ++j) {
      V2<T> t = w16[i * j];
      a[i][j] = cmul<T>(a[i][j], inv ? cconj<T>(t) : t);
    }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    V2<T> b[4] = {a[0][j], a[1][j], a[2][j], a[3][j]};
    dft4<T>(b, inv);
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i * 4 + j] = b[i];
  }
}

struct FftShape {
  int L;        // complex length nlon/2
  int Lp;       // padded row stride in the shared buffers
  int nrad;
  int rad[24];  // radix sequence
};

// One Stockham pass (radix R, Ns = product of earlier radices) over `rows`
// rows held in shared memory; twiddles from the table exp(-2 pi i k / L).
template <typename T, int R>
__device__ void pass_fixed(const V2<T>* in, V2<T>* out, const FftShape& f, int Ns, int rows,
                           const V2<T>* __restrict__ tw, const V2<T>* w16, bool inv) {
  const int nb = f.L / R;
  const int stride = f.L / (Ns * R);
  for (int t = threadIdx.x; t < rows * nb; t += blockDim.x) {
    int g = t / nb, j = t - g * nb;
    const V2<T>* src = in + g * f.Lp;
    V2<T>* dst = out + g * f.Lp;
    int k = j % Ns;
    V2<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        V2<T> w = tw[k * r * stride];
        v[r] = cmul<T>(v[r], inv ? cconj<T>(w) : w);
      }
    }
    if (R == 2) dft2<T>(v);
    if (R == 3) dft3<T>(v, inv);
    if (R == 4) dft4<T>(v, inv);
    if (R == 5) dft5<T>(v, inv);
    if (R == 8) dft8<T>(v, inv);
    if (R == 16) dft16<T>(v, w16, inv);
    int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
  }
}

// Generic odd-prime radix: direct DFT of the twiddled inputs.
template <typename T>
__device__ void pass_generic(const V2<T>* in, V2<T>* out, const FftShape& f, int Ns, int R,
                             int rows, const V2<T>* __restrict__ tw, bool inv) {
  const int nb = f.L / R;
  const int stride = f.L / (Ns * R);
  const int rstride = f.L / R;
  for (int t = threadIdx.x; t < rows * nb; t += blockDim.x) {
    int g = t / nb, j = t - g * nb;
    const V2<T>* src = in + g * f.Lp;
    V2<T>* dst = out + g * f.Lp;
    int k = j % Ns;
    int base = (j / Ns) * Ns * R + k;
    for (int s = 0; s < R; ++s) {
      V2<T> acc = mk2<T>(T(0), T(0));
      for (int r = 0; r < R; ++r) {
        V2<T> v = src[j + r * nb];
        int idx = (k * r * stride + ((r * s) % R) * rstride) % f.L;
        V2<T> w = tw[idx];
        v = cmul<T>(v, inv ? cconj<T>(w) : w);
        acc = cadd<T>(acc, v);
      }
      dst[base + s * Ns] = acc;
    }
  }
}

// Runs the radix sequence; returns the buffer that holds the result.
template <typename T>
__device__ V2<T>* run_passes(V2<T>* a, V2<T>* b, const FftShape& f, int rows,
                             const V2<T>* __restrict__ tw, const V2<T>* w16, bool inv) {
  int Ns = 1;
  for (int p = 0; p < f.nrad; ++p) {
    int R = f.rad[p];
    switch (R) {
      case 2: pass_fixed<T, 2>(a, b, f, Ns, rows, tw, w16, inv); break;
      case 3: pass_fixed<T, 3>(a, b, f, Ns, rows, tw, w16, inv); break;
      case 4: pass_fixed<T, 4>(a, b, f, Ns, rows, tw, w16, inv); break;
      case 5: pass_fixed<T, 5>(a, b, f, Ns, rows, tw, w16, inv); break;
      case 8: pass_fixed<T, 8>(a, b, f, Ns, rows, tw, w16, inv); break;
      case 16: pass_fixed<T, 16>(a, b, f, Ns, rows, tw, w16, inv); break;
      default: pass_generic<T>(a, b, f, Ns, R, rows, tw, inv); break;
    }
    __syncthreads();
    V2<T>* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

struct FoldArgs {
  FftShape f;
  int nlat, nlon, T, H, nlat_odd;
  int G;        // planes per CTA
  int F;        // fields stacked per plane (1 scalar, 2 for (u, v))
  int64_t planes;
};

template <typename T>
__device__ void load_w16(V2<T>* w16, const V2<T>* tw, int L) {
  if (threadIdx.x < 16) {
    // exp(-2 pi i k/16) = tw[k L/16] when 16 | L, else computed
    if (L % 16 == 0) {
      w16[threadIdx.x] = tw[threadIdx.x * (L / 16)];
    } else {
      double s, c;
      sincospi(-2.0 * threadIdx.x / 16.0, &s, &c);
      w16[threadIdx.x] = mk2<T>(T(c), T(s));
    }
  }
}

// grid (planes, nlat, nlon) per field -> waist [m][s][h][r], r = (p*F + f)*2 + c.
template <typename T>
__global__ void forward_fold_kernel(FoldArgs a, const T* __restrict__ g0,
                                    const T* __restrict__ g1, const V2<T>* __restrict__ tw_l,
                                    const V2<T>* __restrict__ tw_n, T* __restrict__ wfold,
                                    float* __restrict__ rowmax) {
  extern __shared__ unsigned char smem_raw[];
  V2<T>* bufA = reinterpret_cast<V2<T>*>(smem_raw);
  const int h = blockIdx.x;
  const int64_t p0 = (int64_t)blockIdx.y * a.G;
  const bool eq = a.nlat_odd && h == a.H - 1;
  const int rpp = eq ? 1 : 2;              // rows per (plane, field)
  const int rows = a.G * a.F * rpp;
  const int Lp = a.f.Lp;
  V2<T>* bufB = bufA + rows * Lp;
  __shared__ V2<T> w16[16];
  load_w16<T>(w16, tw_l, a.f.L);

  // Load rows: row index ((gp*F + f)*rpp + side).
  for (int t = threadIdx.x; t < rows * a.f.L; t += blockDim.x) {
    int row = t / a.f.L, k = t - row * a.f.L;
    int side = row % rpp, pf = row / rpp;
    int f = pf % a.F, gp = pf / a.F;
    int64_t plane = p0 + gp;
    V2<T> v = mk2<T>(T(0), T(0));
    if (plane < a.planes) {
      int j = side ? (a.nlat - 1 - h) : h;
      const T* src = (f ? g1 : g0) + (plane * a.nlat + j) * (int64_t)a.nlon;
      v = reinterpret_cast<const V2<T>*>(src)[k];
    }
    bufA[row * Lp + k] = v;
  }
  __syncthreads();
  V2<T>* Z = run_passes<T>(bufA, bufB, a.f, rows, tw_l, w16, false);

  // Untangle, scale, fold, write.  Thread -> (m, gp, f) with (gp, f) fastest.
  const int L = a.f.L;
  const int nper = a.G * a.F;
  const int64_t R = a.planes * a.F * 2;
  const T inv_n = T(1) / T(a.nlon);
  V2<T>* out = reinterpret_cast<V2<T>*>(wfold);
  float mre = 0.f, mim = 0.f;  // this thread's column maxima (pf = tid % nper)
  for (int t = threadIdx.x; t < (a.T + 1) * nper; t += blockDim.x) {
    int m = t / nper, pf = t - m * nper;
    int gp = pf / a.F;
    if (p0 + gp >= a.planes) continue;
    V2<T> X[2];
    V2<T> w = tw_n[m];
    for (int side = 0; side < rpp; ++side) {
      const V2<T>* zr = Z + (pf * rpp + side) * Lp;
      V2<T> zk = zr[m];
      V2<T> zc = cconj<T>(zr[m == 0 ? 0 : L - m]);
      V2<T> ev = cadd<T>(zk, zc);   // 2 * even part
      V2<T> od = csub<T>(zk, zc);   // 2 * i * odd part
      // X = (ev - i w od) / 2
      V2<T> t1 = cmul<T>(w, od);
      V2<T> xm = mk2<T>(T(0.5) * (ev.x + t1.y), T(0.5) * (ev.y - t1.x));
      X[side] = mk2<T>(xm.x * inv_n, xm.y * inv_n);
    }
    V2<T> S, D;
    if (rpp == 2) {
      S = cadd<T>(X[0], X[1]);
      D = csub<T>(X[0], X[1]);
    } else {
      S = X[0];
      D = mk2<T>(T(0), T(0));
    }
    int64_t rr = (p0 * a.F + pf);  // complex column index = r/2
    int64_t base0 = ((int64_t)(m * 2 + 0) * a.H + h) * (R / 2) + rr;
    int64_t base1 = ((int64_t)(m * 2 + 1) * a.H + h) * (R / 2) + rr;
    out[base0] = S;
    out[base1] = D;
    mre = fmaxf(mre, (float)fmax(fabs(S.x), fabs(D.x)));
    mim = fmaxf(mim, (float)fmax(fabs(S.y), fabs(D.y)));
  }
  if (rowmax != nullptr) {
    const int pf = threadIdx.x % nper;  // fixed per thread: blockDim % nper == 0
    rowmax_merge(rowmax, p0 * a.F + pf, p0 + pf / a.F < a.planes, mre, mim, nper);
  }
}

struct UnfoldArgs {
  FftShape f;
  int nlat, nlon, T, H, nlat_odd;
  int G;
  int mode;
  int64_t planes;
  double radius;
};

// waist(s) -> grid rows.  Waist row index r = (p*F + f)*2 + c with F = 2
// (psi, chi) in the wind mode and F = 1 otherwise.
template <typename T>
__global__ void inverse_unfold_kernel(UnfoldArgs a, const T* __restrict__ wP,
                                      const T* __restrict__ wD, const double* __restrict__ coslat,
                                      const V2<T>* __restrict__ tw_l,
                                      const V2<T>* __restrict__ tw_n, T* __restrict__ out0,
                                      T* __restrict__ out1) {
  extern __shared__ unsigned char smem_raw[];
  V2<T>* bufA = reinterpret_cast<V2<T>*>(smem_raw);
  const int h = blockIdx.x;
  const int64_t p0 = (int64_t)blockIdx.y * a.G;
  const bool eq = a.nlat_odd && h == a.H - 1;
  const int rpp = eq ? 1 : 2;
  const int NO = (a.mode == kUnfoldGradient || a.mode == kUnfoldWind) ? 2 : 1;
  const int FW = a.mode == kUnfoldWind ? 2 : 1;  // fields per plane in the waist
  const int rows = a.G * NO * rpp;
  const int Lp = a.f.Lp;
  const int L = a.f.L;
  V2<T>* bufB = bufA + rows * Lp;
  __shared__ V2<T> w16[16];
  load_w16<T>(w16, tw_l, L);
  const int64_t Rc = a.planes * FW;  // complex columns per waist row block
  const V2<T>* P2 = reinterpret_cast<const V2<T>*>(wP);
  const V2<T>* D2 = reinterpret_cast<const V2<T>*>(wD);
  const T inv_a = T(1.0 / a.radius);

  // Stage 1: Fourier coefficients X_row[m] (m <= T) into bufB, row index
  // ((gp*NO + o)*rpp + side).
  for (int t = threadIdx.x; t < (a.T + 1) * a.G; t += blockDim.x) {
    int m = t / a.G, gp = t - m * a.G;
    int64_t plane = p0 + gp;
    if (plane >= a.planes) continue;
    int j[2] = {h, a.nlat - 1 - h};
    for (int side = 0; side < rpp; ++side) {
      T sgn = side ? T(-1) : T(1);
      T cl = T(coslat[j[side]]);
      T im_over = T(m) / (T(a.radius) * cl);  // m / (a cos phi)
      auto fetch = [&](const V2<T>* w, int f) {
        int64_t c0 = ((int64_t)(m * 2 + 0) * a.H + h) * Rc + plane * FW + f;
        int64_t c1 = ((int64_t)(m * 2 + 1) * a.H + h) * Rc + plane * FW + f;
        V2<T> s = w[c0], d = w[c1];
        return mk2<T>(s.x + sgn * d.x, s.y + sgn * d.y);
      };
      V2<T> o0, o1 = mk2<T>(T(0), T(0));
      if (a.mode == kUnfoldScalar || a.mode == kUnfoldMeridional) {
        o0 = fetch(P2, 0);
      } else if (a.mode == kUnfoldZonal) {
        V2<T> x = fetch(P2, 0);
        o0 = mk2<T>(-T(m) * x.y, T(m) * x.x);
      } else if (a.mode == kUnfoldGradient) {
        V2<T> x = fetch(P2, 0);
        V2<T> y = fetch(D2, 0);
        o0 = mk2<T>(-T(m) * x.y, T(m) * x.x);  // i m X (metric factor after the FFT)
        o1 = y;                                 // dP synthesis (/a after the FFT)
      } else {  // wind: u = -dpsi/a + i m chi/(a cos); v = i m psi/(a cos) + dchi/a
        V2<T> xp = fetch(P2, 0), xc = fetch(P2, 1);
        V2<T> dp = fetch(D2, 0), dc = fetch(D2, 1);
        o0 = mk2<T>(-dp.x * inv_a - im_over * xc.y, -dp.y * inv_a + im_over * xc.x);
        o1 = mk2<T>(-im_over * xp.y + dc.x * inv_a, im_over * xp.x + dc.y * inv_a);
      }
      bufB[((gp * NO + 0) * rpp + side) * Lp + m] = o0;
      if (NO == 2) bufB[((gp * NO + 1) * rpp + side) * Lp + m] = o1;
    }
  }
  __syncthreads();
  // Stage 2: entangle into Z[k], k < L, in bufA.
  for (int t = threadIdx.x; t < rows * L; t += blockDim.x) {
    int row = t / L, k = t - row * L;
    int gp = row / (NO * rpp);
    V2<T> z = mk2<T>(T(0), T(0));
    if (p0 + gp < a.planes) {
      const V2<T>* xr = bufB + row * Lp;
      V2<T> xk = k <= a.T ? xr[k] : mk2<T>(T(0), T(0));
      int kc = L - k;
      V2<T> xc = (k > 0 && kc <= a.T) ? cconj<T>(xr[kc]) : mk2<T>(T(0), T(0));
      if (k == 0) xk.y = T(0);  // irfft reads only the real part of bin 0
      V2<T> s = cadd<T>(xk, xc), d = csub<T>(xk, xc);
      V2<T> w = cconj<T>(tw_n[k]);  // exp(+2 pi i k / N)
      V2<T> wd = cmul<T>(w, d);
      z = mk2<T>(s.x - wd.y, s.y + wd.x);  // s + i w d
    }
    bufA[row * Lp + k] = z;
  }
  __syncthreads();
  V2<T>* zr = run_passes<T>(bufA, bufB, a.f, rows, tw_l, w16, true);

  // Stage 3: write rows with per-row scaling.
  for (int t = threadIdx.x; t < rows * L; t += blockDim.x) {
    int row = t / L, k = t - row * L;
    int side = row % rpp, o = (row / rpp) % NO, gp = row / (NO * rpp);
    int64_t plane = p0 + gp;
    if (plane >= a.planes) continue;
    int j = side ? (a.nlat - 1 - h) : h;
    V2<T> v = zr[row * Lp + k];
    if (a.mode == kUnfoldGradient) {
      if (o == 0) {
        T den = T(a.radius) * T(coslat[j]);
        v.x = v.x / den;
        v.y = v.y / den;
      } else {
        v.x = v.x / T(a.radius);
        v.y = v.y / T(a.radius);
      }
    }
    T* dst = (o ? out1 : out0) + (plane * a.nlat + j) * (int64_t)a.nlon;
    reinterpret_cast<V2<T>*>(dst)[k] = v;
  }
}

__global__ void twiddle_kernel(int L, int N, double2* tl, double2* tn) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < L) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)L, &s, &c);
    tl[k] = make_double2(c, s);
  }
  if (k <= L) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)N, &s, &c);
    tn[k] = make_double2(c, s);
  }
}

__global__ void twiddle_cast_kernel(const double2* in, float2* out, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = make_float2((float)in[k].x, (float)in[k].y);
}

FftShape make_shape(const sht_plan* p) {
  FftShape f{};
  f.L = p->L;
  f.Lp = p->L;
  f.nrad = (int)p->radices.size();
  for (int i = 0; i < f.nrad; ++i) f.rad[i] = p->radices[i];
  return f;
}

template <typename T>
int rows_budget() { return sizeof(T) == 8 ? 4 : 8; }

template <typename T>
size_t smem_bytes(const sht_plan* p, int rows) {
  return (size_t)2 * rows * p->L * sizeof(V2<T>);
}

template <typename K>
void allow_smem(K kernel, size_t bytes) {
  SHT_CUDA_OR_THROW(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)std::max<size_t>(bytes, 48 * 1024)));
}

}  // namespace

void build_fft(sht_plan* p, cudaStream_t s) {
  // Radix plan: 16s, 8, 4, 2, then 3s, 5s, then any other primes.
  int L = p->L;
  std::vector<int> rad;
  int r = L;
  while (r % 16 == 0) { rad.push_back(16); r /= 16; }
  if (r % 8 == 0) { rad.push_back(8); r /= 8; }
  if (r % 4 == 0) { rad.push_back(4); r /= 4; }
  if (r % 2 == 0) { rad.push_back(2); r /= 2; }
  while (r % 3 == 0) { rad.push_back(3); r /= 3; }
  while (r % 5 == 0) { rad.push_back(5); r /= 5; }
  for (int q = 7; r > 1; q += 2)
    while (r % q == 0) { rad.push_back(q); r /= q; }
  SHT_REQUIRE(rad.size() <= 24, "nlon has too many prime factors");
  p->radices = rad;
  p->fast_fft = fast_fft_supported(p) && !p->force_generic_fft;
  if (p->fast_fft) fast_fft_init_constants(s);

  double2 *tl = nullptr, *tn = nullptr;
  SHT_CUDA_OR_THROW(cudaMalloc(&tl, sizeof(double2) * L));
  SHT_CUDA_OR_THROW(cudaMalloc(&tn, sizeof(double2) * (L + 1)));
  twiddle_kernel<<<(L + 256) / 256, 256, 0, s>>>(L, p->nlon, tl, tn);
  SHT_CUDA_OR_THROW(cudaGetLastError());
  if (p->prec == SHT_PREC_F64) {
    p->tw_l = tl;
    p->tw_n = tn;
  } else {
    float2 *fl = nullptr, *fn = nullptr;
    SHT_CUDA_OR_THROW(cudaMalloc(&fl, sizeof(float2) * L));
    SHT_CUDA_OR_THROW(cudaMalloc(&fn, sizeof(float2) * (L + 1)));
    twiddle_cast_kernel<<<(L + 255) / 256, 256, 0, s>>>(tl, fl, L);
    twiddle_cast_kernel<<<(L + 256) / 256, 256, 0, s>>>(tn, fn, L + 1);
    SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
    cudaFree(tl);
    cudaFree(tn);
    p->tw_l = fl;
    p->tw_n = fn;
  }
}

template <typename T>
void launch_forward_fold(const sht_plan* p, const T* g0, const T* g1, int64_t planes,
                         T* wfold, cudaStream_t s, float* rowmax) {
  if constexpr (sizeof(T) == 4) {
    if (p->fast_fft) {
      fast_forward_fold(p, g0, g1, planes, wfold, s, rowmax);
      return;
    }
  }
  // g0 (and g1 for a stacked (u, v) pair) are (planes, nlat, nlon) grids.
  const int fields = g1 ? 2 : 1;
  FoldArgs a{};
  a.f = make_shape(p);
  a.nlat = p->nlat;
  a.nlon = p->nlon;
  a.T = p->T;
  a.H = p->H;
  a.nlat_odd = p->nlat_odd;
  a.F = fields;
  a.G = std::max(1, rows_budget<T>() / (2 * fields));
  a.planes = planes;
  int rows = a.G * a.F * 2;
  size_t sm = smem_bytes<T>(p, rows);
  allow_smem(forward_fold_kernel<T>, sm);
  dim3 grid_dim((unsigned)p->H, (unsigned)div_up(planes, a.G));
  SHT_REQUIRE(rowmax == nullptr || 256 % (a.G * a.F) == 0, "row maxima need 256 % (G F) == 0");
  forward_fold_kernel<T><<<grid_dim, 256, sm, s>>>(a, g0, g1 ? g1 : g0, (const V2<T>*)p->tw_l,
                                                   (const V2<T>*)p->tw_n, wfold, rowmax);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template <typename T>
void launch_inverse_unfold(const sht_plan* p, int mode, const T* wP, const T* wD,
                           int64_t planes, T* out0, T* out1, cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    if (p->fast_fft) {
      fast_inverse_unfold(p, mode, wP, wD, planes, out0, out1, s);
      return;
    }
  }
  UnfoldArgs a{};
  a.f = make_shape(p);
  a.nlat = p->nlat;
  a.nlon = p->nlon;
  a.T = p->T;
  a.H = p->H;
  a.nlat_odd = p->nlat_odd;
  a.mode = mode;
  a.planes = planes;
  a.radius = p->radius;
  int NO = (mode == kUnfoldGradient || mode == kUnfoldWind) ? 2 : 1;
  a.G = std::max(1, rows_budget<T>() / (2 * NO));
  int rows = a.G * NO * 2;
  size_t sm = smem_bytes<T>(p, rows);
  allow_smem(inverse_unfold_kernel<T>, sm);
  dim3 grid_dim((unsigned)p->H, (unsigned)div_up(planes, a.G));
  inverse_unfold_kernel<T><<<grid_dim, 256, sm, s>>>(a, wP, wD, p->d_coslat,
                                                     (const V2<T>*)p->tw_l,
                                                     (const V2<T>*)p->tw_n, out0, out1);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template void launch_forward_fold<float>(const sht_plan*, const float*, const float*, int64_t,
                                         float*, cudaStream_t, float*);
template void launch_forward_fold<double>(const sht_plan*, const double*, const double*, int64_t,
                                          double*, cudaStream_t, float*);
template void launch_inverse_unfold<float>(const sht_plan*, int, const float*, const float*,
                                           int64_t, float*, float*, cudaStream_t);
template void launch_inverse_unfold<double>(const sht_plan*, int, const double*, const double*,
                                            int64_t, double*, double*, cudaStream_t);

}  // namespace sht
