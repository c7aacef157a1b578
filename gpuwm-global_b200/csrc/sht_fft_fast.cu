// Register-resident longitude FFTs for the grid sizes of the ArWen configs
// (nlon = 64 F with F in {2, 3, 4, 6, 8, 12, 16, 24}: 192, 384, 768 and 1536
// longitudes among them), FP32.
//
// One warp owns one grid row.  The complex length L = nlon/2 = 32 F is split
// four-step style as L = F x 32: lane l loads the F samples z[l + 32 j] with F
// independent 8-byte loads issued back to back (the memory-level parallelism
// the shared-memory Stockham kernel lacked), does an F-point DFT in
// registers, applies exp(-+2 pi i l k1 / L), and one padded shared-memory
// transpose hands each of F lanes a 32-point DFT, also in registers.  The
// real-input untangling, 1/nlon scaling and the equator fold (forward) or the
// unfold and the mode combinations (inverse) run in the CTA epilogue /
// prologue, so grid and waist are each touched exactly once.
#include "sht_plan.h"

namespace sht {
namespace {

// exp(-2 pi i k / 24), exp(-2 pi i k / 32) and exp(-2 pi i k / 16), uploaded
// once per process: read as constant-bank operands of the butterfly FMAs.
__constant__ float2 c_w24[24];
__constant__ float2 c_w32[32];
__constant__ float2 c_w16[16];

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconjf(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 caddf(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csubf(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
template <bool INV>
__device__ __forceinline__ float2 rot90f(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
template <bool INV>
__device__ __forceinline__ float2 tw(float2 w) { return INV ? cconjf(w) : w; }

template <bool INV>
__device__ __forceinline__ void d2(float2& a, float2& b) {
  float2 t = a;
  a = caddf(t, b);
  b = csubf(t, b);
}
template <bool INV>
__device__ __forceinline__ void d3(float2& a, float2& b, float2& c) {
  const float s1 = INV ? 0.86602540378443864676f : -0.86602540378443864676f;
  float2 t1 = caddf(b, c), t2 = csubf(b, c);
  float2 m1 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
  float2 m2 = make_float2(-s1 * t2.y, s1 * t2.x);
  a = caddf(a, t1);
  b = caddf(m1, m2);
  c = csubf(m1, m2);
}
template <bool INV>
__device__ __forceinline__ void d4(float2* v) {
  float2 a0 = caddf(v[0], v[2]), a1 = csubf(v[0], v[2]);
  float2 b0 = caddf(v[1], v[3]), b1 = rot90f<INV>(csubf(v[1], v[3]));
  v[0] = caddf(a0, b0);
  v[2] = csubf(a0, b0);
  v[1] = caddf(a1, b1);
  v[3] = csubf(a1, b1);
}
template <bool INV>
__device__ __forceinline__ void d8(float2* v) {
  float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  d4<INV>(e);
  d4<INV>(o);
  const float r = 0.70710678118654752440f;
  o[1] = cmulf(o[1], make_float2(r, INV ? r : -r));
  o[2] = rot90f<INV>(o[2]);
  o[3] = cmulf(o[3], make_float2(-r, INV ? r : -r));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = caddf(e[k], o[k]);
    v[k + 4] = csubf(e[k], o[k]);
  }
}
// Four-step in registers: N = N1 * N2, n = N2 n1 + n2, k = k1 + N1 k2.
template <int N1, bool INV>
__device__ __forceinline__ void dpow2(float2* v) {
  if constexpr (N1 == 1) {
  } else if constexpr (N1 == 2) {
    d2<INV>(v[0], v[1]);
  } else if constexpr (N1 == 4) {
    d4<INV>(v);
  } else if constexpr (N1 == 8) {
    d8<INV>(v);
  } else {  // 16 = 4 x 4
    float2 a[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
      for (int j = 0; j < 4; ++j) a[i][j] = v[j * 4 + i];
      d4<INV>(a[i]);
    }
#pragma unroll
    for (int i = 1; i < 4; ++i)
#pragma unroll
      for (int j = 1; j < 4; ++j) a[i][j] = cmulf(a[i][j], tw<INV>(c_w16[i * j]));
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float2 b[4] = {a[0][j], a[1][j], a[2][j], a[3][j]};
      d4<INV>(b);
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i * 4 + j] = b[i];
    }
  }
}

// F-point DFT, F = P2 (power of two) or 3 * P2.
template <int F, bool INV>
__device__ __forceinline__ void dftF(float2* v) {
  if constexpr (F % 3 != 0) {
    dpow2<F, INV>(v);
  } else {
    constexpr int N1 = F / 3;
    float2 a[3][N1];
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) a[n2][n1] = v[3 * n1 + n2];
      dpow2<N1, INV>(a[n2]);
    }
#pragma unroll
    for (int n2 = 1; n2 < 3; ++n2)
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1) a[n2][k1] = cmulf(a[n2][k1], tw<INV>(c_w24[(n2 * k1 * (24 / F)) % 24]));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      d3<INV>(a[0][k1], a[1][k1], a[2][k1]);
#pragma unroll
      for (int k2 = 0; k2 < 3; ++k2) v[k1 + N1 * k2] = a[k2][k1];
    }
  }
}

// 32-point DFT = 8 x 4.
template <bool INV>
__device__ __forceinline__ void dft32(float2* v) {
  float2 a[4][8];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) a[n2][n1] = v[4 * n1 + n2];
    d8<INV>(a[n2]);
  }
#pragma unroll
  for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
    for (int k1 = 1; k1 < 8; ++k1) a[n2][k1] = cmulf(a[n2][k1], tw<INV>(c_w32[n2 * k1]));
#pragma unroll
  for (int k1 = 0; k1 < 8; ++k1) {
    float2 b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    d4<INV>(b);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 8 * k2] = b[k2];
  }
}

// Per-warp shared region: F rows of 33 (the transpose), reused as the
// natural-order spectrum of L = 32 F entries.  Regions are padded to 2 float2
// modulo 8, so that the fold/unfold loops, in which lanes 4j..4j+3 touch the
// same order m of four different rows, hit four distinct bank groups.
template <int F> struct WarpSmem {
  static constexpr int kStride = 33;
  static constexpr int kFloats2 = F * kStride + ((2 - (F * kStride) % 8) + 8) % 8;
};

// The four-step twiddles exp(-2 pi i l k1 / L) of every lane l, as a shared
// table [k1][32]: a warp's read of one k1 is 32 consecutive entries (two
// wavefronts), where reading them from the length-L table in global memory
// touched up to F * 8 different cache lines per instruction.
template <int F>
__device__ __forceinline__ void load_lane_twiddles(float2* tws, const float2* __restrict__ twL) {
  constexpr int L = 32 * F;
  for (int e = threadIdx.x; e < F * 32; e += blockDim.x) {
    const int k1 = e >> 5, l = e & 31;
    tws[e] = twL[(l * k1) % L];
  }
}

// R rows per warp: for small F one row leaves most lanes idle in the
// 32-point stage (F of 32), so a warp takes R rows, the largest power of two
// with R x F <= 24 (16 to 24 busy lanes; a power of two so that a CTA's
// column count stays a divisor of 32).  Row r's
// registers z[r][j] = x_r[l + 32 j]; its shared slot is reg + r * slot (the
// slot's first F x 33 entries hold the transpose, then the natural-order
// spectrum).  With `out`, row r's spectrum goes straight from the 32-point
// DFT's registers to out + r * out_stride instead of to its slot.
template <int F> struct RowsPerWarp {
  static constexpr int R = 24 / F >= 8 ? 8 : (24 / F >= 4 ? 4 : (24 / F >= 2 ? 2 : 1));
};

template <int F, int R, bool INV, bool UNIFORM>
__device__ __forceinline__ void warp_fft_rows(float2 (&z)[R][F], float2* reg, int slot,
                                              const float2* tws, int lane,
                                              float2* __restrict__ out = nullptr,
                                              int64_t out_stride = 0, int nvalid = R) {
  constexpr int NL = R * F;  // lanes busy in the 32-point stage
#pragma unroll
  for (int r = 0; r < R; ++r) dftF<F, INV>(z[r]);
  // exp(-+2 pi i lane k1 / L), one table read for all R rows
#pragma unroll
  for (int k1 = 1; k1 < F; ++k1) {
    const float2 w = tw<INV>(tws[k1 * 32 + lane]);
#pragma unroll
    for (int r = 0; r < R; ++r) z[r][k1] = cmulf(z[r][k1], w);
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int k1 = 0; k1 < F; ++k1) reg[r * slot + k1 * WarpSmem<F>::kStride + lane] = z[r][k1];
  __syncwarp();
  // lane -> (row r2, column kk) of the transpose.  Lanes >= NL repeat a busy
  // lane's column (UNIFORM) and drop the result: a branch around the whole
  // 32-point DFT costs ~70 registers once the row pass sits inside a loop.
  // For NL > 16 they take lanes NL-16 .. 15, whose banks differ from those
  // of lanes 16 .. NL-1 read by the same half-warp.
  const int lr = lane < NL ? lane : (NL > 16 ? lane - 16 : lane % NL);
  const int r2 = lr / F, kk = lr - r2 * F;
  const float2* col = reg + r2 * slot + kk * WarpSmem<F>::kStride;
  float2 y[32];
  if constexpr (UNIFORM) {
#pragma unroll
    for (int l = 0; l < 32; ++l) y[l] = col[l];
    __syncwarp();
    dft32<INV>(y);
  } else {
    if (lane < NL) {
#pragma unroll
      for (int l = 0; l < 32; ++l) y[l] = col[l];
    }
    __syncwarp();
    if (lane < NL) dft32<INV>(y);
  }
  // output index k = kk + F k2 (natural order) of row r2
  if (out != nullptr) {
    if (lane < NL && r2 < nvalid) {
      float2* o = out + r2 * out_stride + kk;
#pragma unroll
      for (int k2 = 0; k2 < 32; ++k2) __stcs(o + F * k2, y[k2]);
    }
    return;
  }
  if (lane < NL) {
    float2* o = reg + r2 * slot + kk;
#pragma unroll
    for (int k2 = 0; k2 < 32; ++k2) o[F * k2] = y[k2];
  }
  __syncwarp();
}

// The L-point complex FFT of one warp's row: in registers z[j] = x[l + 32 j]
// (lane l); out: the natural-order spectrum written to `reg` (length L).
template <int F, bool INV>
__device__ __forceinline__ void warp_fft(float2 (&z)[F], float2* reg, const float2* tws, int lane) {
  float2(&z1)[1][F] = *reinterpret_cast<float2(*)[1][F]>(&z);
  warp_fft_rows<F, 1, INV, false>(z1, reg, 0, tws, lane);
}

// A CTA runs kWarps warps, one grid row each: G planes x NF fields x the two
// hemisphere rows (8 rows).
constexpr int kWarps = 8;

// An opaque copy of a pointer.  The inverse kernel reads its entangling
// twiddles through it, so the compiler cannot hoist a whole row of them into
// registers ahead of the butterflies (~20 registers per thread, one resident
// CTA per SM fewer).
__device__ __forceinline__ const float2* opaque(const float2* p) {
  asm volatile("" : "+l"(p));
  return p;
}

struct FastFoldArgs {
  int nlat, nlon, T, H, nlat_odd, F, G;  // F: fields per plane; G: planes per CTA
  int64_t planes;
  int pf_dist;  // latitude pairs ahead whose rows a CTA prefetches into L2 (0: none)
};

// Bulk prefetch of a contiguous global range into L2 (16-byte aligned, a
// multiple of 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// grid -> waist [m][s][h][r], r = (p*F + f)*2 + c.  A CTA of W warps holds
// W x R row slots, slot s = q * 2 + side for column q = gp*F + f (plane gp of
// the CTA's block, field f); warp w transforms slots w, w + W, ... (R rows,
// all on one side).
template <int FF, int W, int TC>
__global__ void __launch_bounds__(W * 32, 24 / W) fast_forward_fold(FastFoldArgs a,
                                                                    const float* __restrict__ g0,
                                                                    const float* __restrict__ g1,
                                                                    const float2* __restrict__ twL,
                                                                    const float2* __restrict__ twN,
                                                                    float2* __restrict__ wfold,
                                                                    float* __restrict__ rowmax) {
  constexpr int L = 32 * FF;
  constexpr int R = RowsPerWarp<FF>::R;
  constexpr int SL = WarpSmem<FF>::kFloats2;  // floats2 per row slot
  extern __shared__ float2 smem_dyn[];
  auto smem = [&](int slot) { return smem_dyn + slot * SL; };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Plane blocks vary fastest over the grid: CTAs that run together touch
  // adjacent slices of every waist row.
  const int h = blockIdx.y;
  const int64_t p0 = (int64_t)blockIdx.x * a.G;
  const bool eq = a.nlat_odd && h == a.H - 1;
  // Columns per CTA: W / 2 x R (a compile-time divisor in the loops below).
  constexpr int nper = W / 2 * R;
  const int fsh = a.F == 2 ? 1 : 0;  // log2 of the field count
  float2* tws = smem_dyn + W * R * SL;
  float2* twn = tws + FF * 32;  // the untangling twiddles exp(-2 pi i m / nlon), m <= T
  // The rows of the CTA about one resident wave later (same plane block,
  // pf_dist latitude pairs on) are pulled into L2 now, so that CTA's loads
  // hit L2 instead of waiting on DRAM at its start.
  if (a.pf_dist > 0 && threadIdx.x < W * R) {
    const int hp = h + a.pf_dist;
    const int q2 = threadIdx.x >> 1, sd2 = threadIdx.x & 1;
    const int64_t pl2 = p0 + (q2 >> fsh);
    if (hp < a.H && pl2 < a.planes && !(a.nlat_odd && hp == a.H - 1 && sd2 == 1)) {
      const int j2 = sd2 ? (a.nlat - 1 - hp) : hp;
      prefetch_l2(((q2 & (a.F - 1)) ? g1 : g0) + (pl2 * a.nlat + j2) * (int64_t)a.nlon,
                  (uint32_t)(a.nlon * sizeof(float)));
    }
  }
  load_lane_twiddles<FF>(tws, twL);
  for (int m = threadIdx.x; m <= a.T; m += blockDim.x) twn[m] = twN[m];
  __syncthreads();
  {
    float2 z[R][FF];
    const int side = warp & 1;  // W is even: every slot w + W r has this side
    const int j = side ? (a.nlat - 1 - h) : h;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int q = (warp + W * r) >> 1;
      const int f = q & (a.F - 1);
      const int64_t plane = p0 + (q >> fsh);
      if (plane < a.planes && !(eq && side == 1)) {
        const float2* src =
            reinterpret_cast<const float2*>((f ? g1 : g0) + (plane * a.nlat + j) * (int64_t)a.nlon);
#pragma unroll
        for (int i = 0; i < FF; ++i) z[r][i] = __ldcs(src + lane + 32 * i);
      } else {
#pragma unroll
        for (int i = 0; i < FF; ++i) z[r][i] = make_float2(0.f, 0.f);
      }
    }
    warp_fft_rows<FF, R, false, false>(z, smem(warp), W * SL, tws, lane);
  }
  __syncthreads();
  // Untangle, scale, fold, write.
  // 0.5 / nlon: (x / 2) / nlon and x * (0.5 / nlon) round alike (both
  // scalings by 2 are exact).
  const float half_inv_n = 0.5f / (float)a.nlon;
  const int64_t Rc = a.planes * a.F;  // complex columns per waist row
  float mre = 0.f, mim = 0.f;         // this thread's column maxima
  const int T = TC >= 0 ? TC : a.T;   // compile-time on the linear grid
  // Thread -> column q (fixed: blockDim is a multiple of nper) and orders
  // m0, m0 + mstep, ...; the waist pointers advance by a constant stride.
  const int q = threadIdx.x % nper;
  const int mstep = (W * 32) / nper;
  if (p0 + (q >> fsh) < a.planes) {
    const float2* zr0 = smem(q * 2);
    const float2* zr1 = smem(q * 2 + 1);
    const int64_t dsd = (int64_t)a.H * Rc;  // S row -> D row of the same order
    const int64_t dm = (int64_t)(2 * mstep) * dsd;
    float2* dst = wfold + ((int64_t)(2 * (threadIdx.x / nper)) * a.H + h) * Rc + p0 * a.F + q;
    for (int m = threadIdx.x / nper; m <= T; m += mstep, dst += dm) {
      const float2 w = twn[m];
      const int mc = m == 0 ? 0 : L - m;
      float2 X[2];
#pragma unroll
      for (int sd = 0; sd < 2; ++sd) {
        if (sd == 1 && eq) {
          X[1] = make_float2(0.f, 0.f);
          continue;
        }
        const float2* zr = sd ? zr1 : zr0;
        const float2 zk = zr[m], zc = cconjf(zr[mc]);
        const float2 ev = caddf(zk, zc), od = csubf(zk, zc);
        const float2 t1 = cmulf(w, od);
        X[sd] = make_float2((ev.x + t1.y) * half_inv_n, (ev.y - t1.x) * half_inv_n);
      }
      const float2 S = eq ? X[0] : caddf(X[0], X[1]);
      const float2 D = eq ? make_float2(0.f, 0.f) : csubf(X[0], X[1]);
      __stcs(dst, S);
      __stcs(dst + dsd, D);
      mre = fmaxf(mre, fmaxf(fabsf(S.x), fabsf(D.x)));
      mim = fmaxf(mim, fmaxf(fabsf(S.y), fabsf(D.y)));
    }
  }
  if (rowmax != nullptr) {
    rowmax_merge(rowmax, p0 * a.F + q, p0 + (q >> fsh) < a.planes, mre, mim, nper);
  }
}

struct FastUnfoldArgs {
  int nlat, nlon, T, H, nlat_odd, mode, G;
  int64_t planes;
  float radius;
};

// waist(s) -> grid.  Warp w handles (row pair index po = w >> 1, side = w & 1)
// with po = gp*NO + o (o: output field).  NF waist columns feed each
// (m, plane): 1 (scalar, zonal, meridional), 2 (gradient: the P and dP
// syntheses of one field), 4 (wind: P and dP of psi and chi).
template <int FF, int NF>
__global__ void __launch_bounds__(kWarps * 32) fast_inverse_unfold(FastUnfoldArgs a,
                                                                   const float2* __restrict__ wP,
                                                                   const float2* __restrict__ wD,
                                                                   const double* __restrict__ coslat,
                                                                   const float2* __restrict__ twL,
                                                                   const float2* __restrict__ twN,
                                                                   float* __restrict__ out0,
                                                                   float* __restrict__ out1) {
  constexpr int L = 32 * FF;
  constexpr int NO = NF == 1 ? 1 : 2;
  extern __shared__ float2 smem_dyn[];
  auto smem = [&](int w) { return smem_dyn + w * WarpSmem<FF>::kFloats2; };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Plane blocks vary fastest over the grid: CTAs that run together touch
  // adjacent slices of every waist row.
  const int h = blockIdx.y;
  const int64_t p0 = (int64_t)blockIdx.x * a.G;
  const bool eq = a.nlat_odd && h == a.H - 1;
  const int64_t Rc = a.planes * (NF == 4 ? 2 : 1);
  const float inv_a = 1.0f / a.radius;
  const int jmir = a.nlat - 1 - h;  // the mirror row (side 1)

  float2* tws = smem_dyn + kWarps * WarpSmem<FF>::kFloats2;
  load_lane_twiddles<FF>(tws, twL);
  // Stage 1: Fourier coefficients of every output row into smem[row][m].
  // Each thread first issues the waist loads of kBatch items (NF symmetric /
  // antisymmetric pairs each), then combines them: the loads of a batch are
  // in flight together instead of one dependent round trip per item.
  constexpr int kBatch = NF == 4 ? 2 : 4;
  constexpr int G = kWarps / 2 / NO;  // planes per CTA
  const int total = (a.T + 1) * G;
  for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
    float2 S[kBatch][NF], D[kBatch][NF];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int t = base + u * blockDim.x;
      const int m = t / G, gp = t - m * G;
      if (t < total && p0 + gp < a.planes) {
        const int64_t r = (p0 + gp) * (NF == 4 ? 2 : 1);
        const int64_t c0 = ((int64_t)(m * 2 + 0) * a.H + h) * Rc + r;
        const int64_t c1 = ((int64_t)(m * 2 + 1) * a.H + h) * Rc + r;
#pragma unroll
        for (int k = 0; k < NF; ++k) {
          const float2* w = (NF == 1 || k < NF / 2) ? wP : wD;
          const int fld = NF == 4 ? (k & 1) : 0;
          S[u][k] = __ldcs(w + c0 + fld);
          D[u][k] = __ldcs(w + c1 + fld);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int t = base + u * blockDim.x;
      const int m = t / G, gp = t - m * G;
      if (t >= total || p0 + gp >= a.planes) continue;
#pragma unroll
      for (int sd = 0; sd < 2; ++sd) {
        if (sd == 1 && eq) continue;
        const float sgn = sd ? -1.f : 1.f;
        float2 x[NF];
#pragma unroll
        for (int k = 0; k < NF; ++k)
          x[k] = make_float2(S[u][k].x + sgn * D[u][k].x, S[u][k].y + sgn * D[u][k].y);
        float2 o0, o1 = make_float2(0.f, 0.f);
        if constexpr (NF == 1) {
          o0 = a.mode == kUnfoldZonal ? make_float2(-(float)m * x[0].y, (float)m * x[0].x) : x[0];
        } else if constexpr (NF == 2) {
          o0 = make_float2(-(float)m * x[0].y, (float)m * x[0].x);
          o1 = x[1];
        } else {
          // x = {P psi, P chi, dP psi, dP chi}
          const float im_over = (float)m / (a.radius * (float)coslat[sd ? jmir : h]);
          o0 = make_float2(-x[2].x * inv_a - im_over * x[1].y, -x[2].y * inv_a + im_over * x[1].x);
          o1 = make_float2(-im_over * x[0].y + x[3].x * inv_a, im_over * x[0].x + x[3].y * inv_a);
        }
        smem((gp * NO + 0) * 2 + sd)[m] = o0;
        if (NO == 2) smem((gp * NO + 1) * 2 + sd)[m] = o1;
      }
    }
  }
  __syncthreads();
  const int po = warp >> 1, side = warp & 1;
  const int o = po % NO, gp = po / NO;
  const int64_t plane = p0 + gp;
  if (po >= G * NO || plane >= a.planes || (eq && side == 1)) return;
  float2* reg = smem(warp);
  const float2* tn = opaque(twN);
  // Stage 2: entangle z[k] for k = lane + 32 j straight into registers.
  float2 z[FF];
#pragma unroll
  for (int i = 0; i < FF; ++i) {
    int k = lane + 32 * i;
    float2 xk = k <= a.T ? reg[k] : make_float2(0.f, 0.f);
    int kc = L - k;
    float2 xc = (k > 0 && kc <= a.T) ? cconjf(reg[kc]) : make_float2(0.f, 0.f);
    if (k == 0) xk.y = 0.f;
    float2 s = caddf(xk, xc), d = csubf(xk, xc);
    float2 wd = cmulf(cconjf(tn[k]), d);
    z[i] = make_float2(s.x - wd.y, s.y + wd.x);
  }
  __syncwarp();
  warp_fft<FF, true>(z, reg, tws, lane);
  // Stage 3: natural-order z[n] -> x[2n], x[2n+1] with the row scaling.
  const int j = side ? jmir : h;
  // The gradient divides the grid by (a cos phi) and by a, as the reference does.
  const bool divide = NF == 2;
  const float den = o == 0 ? a.radius * (float)coslat[j] : a.radius;
  float2* dst = reinterpret_cast<float2*>((o ? out1 : out0) + (plane * a.nlat + j) * (int64_t)a.nlon);
#pragma unroll 4
  for (int i = 0; i < FF; ++i) {
    float2 v = reg[lane + 32 * i];
    if (divide) v = make_float2(v.x / den, v.y / den);
    __stcs(dst + lane + 32 * i, v);
  }
}

// The scalar inverse (one waist column per plane: scalar, zonal, meridional)
// as a persistent kernel: each CTA walks a strided list of items (4 planes x
// one latitude pair), and the waist slices of its next item stream into a
// shared staging buffer with cp.async (no registers held) while the warps
// FFT the current one.  Only a CTA's first item exposes the gather latency.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// FFT and store this warp's R rows: slot reg + r * slot holds row r's
// entangled sequence Z[0..L) in natural order (written by the unfold pass);
// output rows out_row0 + r * out_stride floats2, the first `nvalid` stored.
template <int FF, int R>
__device__ __forceinline__ void inverse_rows_out(float2* reg, int slot, const float2* tws,
                                                 float2* __restrict__ out_row0, int64_t out_stride,
                                                 int lane, int nvalid) {
  float2 z[R][FF];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < FF; ++i) z[r][i] = reg[r * slot + lane + 32 * i];
  __syncwarp();
  warp_fft_rows<FF, R, true, true>(z, reg, slot, tws, lane, out_row0, out_stride, nvalid);
  __syncwarp();  // every lane's reads of reg are done before the next item's unfold
}

// Persistent inverse over items of one latitude pair: NF waist columns per
// plane (1: scalar/zonal/meridional; 2: gradient, the P and dP syntheses of
// one field; 4: wind, P and dP of psi and chi) and NO = 1 or 2 output fields.
// An item holds G planes (2 for NF = 1, 2; 1 for NF = 4), so every waist
// slice it needs is one 16-byte chunk per (buffer, S/D, order): two planes,
// or psi and chi of one plane.  2 x G x NO warps, one output row (plane,
// field, side) each.  TC >= 0: the truncation as a compile-time constant
// (the linear grid, T + 1 = 2 nlon / 3), which fixes every order bound.
template <int NF> struct InvCfg {
  static constexpr int NO = NF == 1 ? 1 : 2;  // output fields
  static constexpr int NB = NF == 1 ? 1 : 2;  // waist buffers (P, dP)
  static constexpr int G = NF == 4 ? 1 : 2;   // planes per warp row group
  static constexpr int W = 2 * G * NO;        // warps
};

template <int FF, int NF, int TC>
__global__ void __launch_bounds__(InvCfg<NF>::W * 32, 16 / InvCfg<NF>::W)
    fast_inverse_pair(FastUnfoldArgs a, const float2* __restrict__ wP,
                      const float2* __restrict__ wD, const double* __restrict__ coslat,
                      const float2* __restrict__ twL, const float2* __restrict__ twN,
                      float* __restrict__ out0, float* __restrict__ out1, int n_pb) {
  constexpr int NO = InvCfg<NF>::NO, NB = InvCfg<NF>::NB, kW = InvCfg<NF>::W;
  constexpr int R = RowsPerWarp<FF>::R;     // rows per warp
  constexpr int GI = InvCfg<NF>::G * R;      // planes per item
  constexpr int CW = NF == 4 ? 2 * GI : GI;  // waist columns per item (even)
  constexpr int SL = WarpSmem<FF>::kFloats2;
  constexpr int L = 32 * FF;  // complex row length (nlon / 2)
  extern __shared__ float2 smem_dyn[];
  auto rows = [&](int slot) { return smem_dyn + slot * SL; };
  float2* tws = smem_dyn + kW * R * SL;
  float2* twn = tws + FF * 32;    // the entangling twiddles exp(-2 pi i k / nlon), k < L
  float2* stage = twn + 32 * FF;  // [buffer][s][m][CW] waist slices of the item in flight
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t Rc = NF == 4 ? 2 * a.planes : a.planes;  // waist columns per row
  const int nms = 2 * (a.T + 1);
  const int64_t n_items = (int64_t)n_pb * a.H;
  // Item i: plane block i % n_pb (fastest: CTAs that run together touch
  // adjacent slices of every waist row), latitude pair i / n_pb.
  auto prefetch = [&](int64_t item) {
    const int h = (int)(item / n_pb);
    const int64_t p0 = (item - (int64_t)h * n_pb) * GI;
    const int64_t c0 = NF == 4 ? 2 * p0 : p0;  // first waist column
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const float2* w = b ? wD : wP;
      for (int e = threadIdx.x; e < nms * (CW / 2); e += blockDim.x) {
        const int c = e % (CW / 2), ms = e / (CW / 2);  // compile-time divisor
        const int64_t valid = Rc - (c0 + 2 * c);  // columns that exist from this chunk on
        const uint32_t bytes = valid >= 2 ? 16u : (valid == 1 ? 8u : 0u);
        const float2* src = bytes ? w + ((int64_t)ms * a.H + h) * Rc + c0 + 2 * c : wP;
        // S (s = 0) and D (s = 1) in separate halves, orders contiguous.
        cp_async16(stage + ((b * 2 + (ms & 1)) * (a.T + 1) + (ms >> 1)) * CW + 2 * c, src, bytes);
      }
    }
    cp_async_commit();
  };
  int64_t item = blockIdx.x;
  if (item < n_items) prefetch(item);
  load_lane_twiddles<FF>(tws, twL);
  for (int k = threadIdx.x; k < 32 * FF; k += blockDim.x) twn[k] = twN[k];
  // warp w: slots w, w + kW, ...; slot s = (gg * NO + o) * 2 + side
  const int side = warp & 1, o = (warp >> 1) % NO, gp = (warp >> 1) / NO;
  const float inv_a = 1.0f / a.radius;
  for (; item < n_items; item += gridDim.x) {
    const int h = (int)(item / n_pb);
    const int64_t p0 = (item - (int64_t)h * n_pb) * GI;
    const bool eq = a.nlat_odd && h == a.H - 1;
    const int jmir = a.nlat - 1 - h;  // the mirror row (side 1)
    cp_async_wait_all();
    __syncthreads();  // the item's slices landed; every warp stored its previous rows
    const int T = TC >= 0 ? TC : a.T;
    const int T1 = T + 1;
    // Row scale factors of the two sides: 1 / (a cos phi) (gradient, wind).
    float ie[2] = {0.f, 0.f};
    if constexpr (NF != 1) {
      ie[0] = 1.0f / (a.radius * (float)coslat[h]);
      ie[1] = 1.0f / (a.radius * (float)coslat[jmir]);
    }
    // x[o][sd]: the spectrum of order j (j <= T) of output field o on side
    // sd, from the symmetric and antisymmetric parts of plane g.
    auto order_values = [&](int j, int g, float2 (&x)[NO][2]) {
      float2 S[NF], D[NF];
#pragma unroll
      for (int k = 0; k < NF; ++k) {
        const int b = NF == 1 ? 0 : (NF == 2 ? k : k >> 1);
        const int c = NF == 4 ? 2 * g + (k & 1) : g;
        S[k] = stage[((b * 2 + 0) * T1 + j) * CW + c];
        D[k] = stage[((b * 2 + 1) * T1 + j) * CW + c];
      }
      const float mf = (float)j;
#pragma unroll
      for (int sd = 0; sd < 2; ++sd) {
        const float sgn = sd ? -1.f : 1.f;
        float2 v[NF];
#pragma unroll
        for (int k = 0; k < NF; ++k) v[k] = make_float2(S[k].x + sgn * D[k].x, S[k].y + sgn * D[k].y);
        if constexpr (NF == 1) {
          x[0][sd] = a.mode == kUnfoldZonal ? make_float2(-mf * v[0].y, mf * v[0].x) : v[0];
        } else if constexpr (NF == 2) {
          // gradient: (i m P) / (a cos phi) east, (dP) / a north; the
          // divisions applied here, ahead of the (linear) FFT
          x[0][sd] = make_float2(-mf * v[0].y * ie[sd], mf * v[0].x * ie[sd]);
          x[1][sd] = make_float2(v[1].x * inv_a, v[1].y * inv_a);
        } else {
          // v = {P psi, P chi, dP psi, dP chi}
          const float im_over = mf * ie[sd];
          x[0][sd] = make_float2(-v[2].x * inv_a - im_over * v[1].y, -v[2].y * inv_a + im_over * v[1].x);
          x[1][sd] = make_float2(-im_over * v[0].y + v[3].x * inv_a, im_over * v[0].x + v[3].y * inv_a);
        }
      }
    };
    // Entangle into the rows: Z[k] = A + conj(C) + i conj(w_k) (A - conj(C))
    // with A = X[k], C = X[L - k], w_k = exp(-2 pi i k / nlon), for the
    // half-length complex FFT of the real row.  Z[L - k] takes the same A, C
    // and w_k (w_{L-k} = -conj(w_k)): with sm = A + conj(C) and
    // t = conj(w_k)(A - conj(C)), Z[k] = sm + i t and Z[L - k] = conj(sm) + i conj(t).
    auto entangle = [&](int g, int k, const float2 (&A)[NO][2], const float2 (&C)[NO][2], float2 w,
                        bool pair) {
#pragma unroll
      for (int o = 0; o < NO; ++o)
#pragma unroll
        for (int sd = 0; sd < 2; ++sd) {
          if (sd == 1 && eq) continue;
          float2* row = rows((g * NO + o) * 2 + sd);
          const float2 p = A[o][sd], q = C[o][sd];
          const float2 sm = make_float2(p.x + q.x, p.y - q.y), df = make_float2(p.x - q.x, p.y + q.y);
          const float2 t = cmulf(cconjf(w), df);
          row[k] = make_float2(sm.x - t.y, sm.y + t.x);
          if (pair) row[L - k] = make_float2(sm.x + t.y, t.x - sm.y);
        }
    };
    // Thread -> (k, plane g), k < L / 2: Z[k] and Z[L - k]; k = 0 also
    // writes the self-paired middle entry Z[L / 2].
    for (int t = threadIdx.x; t < (L / 2) * GI; t += blockDim.x) {
      const int k = t / GI, g = t - k * GI;  // GI: a compile-time power of two
      if (p0 + g >= a.planes) continue;
      const int kc = L - k;
      float2 A[NO][2], C[NO][2];
      if (k <= T) {
        order_values(k, g, A);
      } else {
#pragma unroll
        for (int o = 0; o < NO; ++o) A[o][0] = A[o][1] = make_float2(0.f, 0.f);
      }
      if (k > 0 && kc <= T) {
        order_values(kc, g, C);
      } else {
#pragma unroll
        for (int o = 0; o < NO; ++o) C[o][0] = C[o][1] = make_float2(0.f, 0.f);
      }
      if (k == 0) {
        // order 0 is real; its partner L lies outside the row
#pragma unroll
        for (int o = 0; o < NO; ++o) A[o][0].y = A[o][1].y = 0.f;
      }
      entangle(g, k, A, C, twn[k], k > 0);
      if (k == 0) {
        float2 M[NO][2];
        if (L / 2 <= T) {
          order_values(L / 2, g, M);
        } else {
#pragma unroll
          for (int o = 0; o < NO; ++o) M[o][0] = M[o][1] = make_float2(0.f, 0.f);
        }
        entangle(g, L / 2, M, M, twn[L / 2], false);
      }
    }
    __syncthreads();  // the staging buffer is free again
    if (item + gridDim.x < n_items) prefetch(item + gridDim.x);
    const int64_t plane = p0 + gp;  // the warp's first row; the others are GI / R apart
    // The lane index, made opaque per item: the per-lane masks and offsets of
    // the row pass are rebuilt every item instead of held across the loop.
    int ln = lane;
    asm volatile("" : "+r"(ln));
    if (plane < a.planes && !(eq && side == 1)) {
      constexpr int G = InvCfg<NF>::G;
      float* out = o ? out1 : out0;
      float2* row0 = reinterpret_cast<float2*>(out + (plane * a.nlat + (side ? jmir : h)) * (int64_t)a.nlon);
      const int64_t stride = (int64_t)G * a.nlat * a.nlon / 2;  // floats2 between the warp's rows
      // rows past the plane count are transformed but not stored
      const int64_t left = (a.planes - plane + G - 1) / G;
      const int nvalid = left < R ? (int)left : R;
      inverse_rows_out<FF, R>(rows(warp), kW * SL, tws, row0, stride, ln, nvalid);
    }
  }
}

// SMs of the current device, and resident CTAs per SM of a kernel with the
// given block and dynamic shared memory (the latter also raised to `sm`).
int sm_count() {
  int dev = 0, sms = 0;
  SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
  SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return sms;
}
template <typename K>
int resident_ctas(K kernel, int threads, size_t sm) {
  SHT_CUDA_OR_THROW(
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int per_sm = 0;
  SHT_CUDA_OR_THROW(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, sm));
  SHT_REQUIRE(per_sm > 0, "FFT kernel does not fit on an SM");
  return per_sm;
}

// The waist rows must be 16-byte aligned for cp.async: an even plane count.
// One persistent CTA per resident slot.
template <int FF, int NF, int TC>
void launch_inv_pair_t(const sht_plan* p, int mode, const float* wP, const float* wD,
                       int64_t planes, float* out0, float* out1, cudaStream_t s) {
  constexpr int kW = InvCfg<NF>::W, NB = InvCfg<NF>::NB, R = RowsPerWarp<FF>::R;
  constexpr int GI = InvCfg<NF>::G * R, CW = NF == 4 ? 2 * GI : GI;
  FastUnfoldArgs a{p->nlat, p->nlon, p->T, p->H, p->nlat_odd ? 1 : 0, mode, GI, planes,
                   (float)p->radius};
  const int n_pb = (int)div_up(planes, GI);
  const size_t sm = sizeof(float2) * (kW * R * WarpSmem<FF>::kFloats2 + 2 * FF * 32 +
                                      (size_t)NB * 2 * (p->T + 1) * CW);
  const int64_t n_items = (int64_t)n_pb * p->H;
  if (n_items == 0) return;
  const int64_t ctas = std::min<int64_t>(
      n_items, (int64_t)resident_ctas(fast_inverse_pair<FF, NF, TC>, kW * 32, sm) * sm_count());
  fast_inverse_pair<FF, NF, TC><<<(unsigned)ctas, kW * 32, sm, s>>>(
      a, (const float2*)wP, (const float2*)(wD ? wD : wP), p->d_coslat, (const float2*)p->tw_l,
      (const float2*)p->tw_n, out0, out1 ? out1 : out0, n_pb);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}
// The waist rows must be 16-byte aligned for cp.async: for NF = 1, 2 (one
// waist column per plane) an even plane count; NF = 4 (two per plane) any.
template <int FF, int NF>
void launch_inv_pair(const sht_plan* p, int mode, const float* wP, const float* wD,
                     int64_t planes, float* out0, float* out1, cudaStream_t s) {
  // The linear grid's truncation, T + 1 = 2 nlon / 3 = 64 F / 3, when it is whole.
  constexpr int TLIN = (64 * FF) % 3 == 0 ? 64 * FF / 3 - 1 : -1;
  if (TLIN >= 0 && p->T == TLIN)
    launch_inv_pair_t<FF, NF, TLIN>(p, mode, wP, wD, planes, out0, out1, s);
  else
    launch_inv_pair_t<FF, NF, -1>(p, mode, wP, wD, planes, out0, out1, s);
}

// L2 prefetch of the rows one resident wave ahead in the forward FFT.
constexpr bool kFwdPrefetch = true;
// Warps per CTA of the forward FFT.  Eight: each CTA then writes 32-byte
// (full-sector) pieces of every waist row; four (16-byte pieces, six CTAs
// per SM) measured 0.72 ms against 0.43 ms at T511 x 200 planes.
constexpr int kFwdWarps = 8;
template <int FF, int TC>
void launch_fwd_t(const sht_plan* p, const float* g0, const float* g1, int64_t planes,
                  float* wfold, cudaStream_t s, float* rowmax) {
  constexpr int W = kFwdWarps;
  constexpr int R = RowsPerWarp<FF>::R;
  FastFoldArgs a{p->nlat, p->nlon, p->T, p->H, p->nlat_odd ? 1 : 0, g1 ? 2 : 1, 0, planes, 0};
  a.G = W / 2 * R / a.F;  // planes per CTA
  dim3 grid((unsigned)div_up(planes, a.G), (unsigned)p->H);
  const size_t sm = sizeof(float2) * (W * R * WarpSmem<FF>::kFloats2 + FF * 32 + p->T + 1);
  // One resident wave of CTAs, in latitude pairs (grid.x CTAs per pair);
  // resident_ctas also raises the kernel's shared-memory limit to `sm`.
  const int64_t wave = (int64_t)resident_ctas(fast_forward_fold<FF, W, TC>, W * 32, sm) * sm_count();
  a.pf_dist = kFwdPrefetch ? (int)div_up(wave, (int64_t)grid.x) : 0;
  fast_forward_fold<FF, W, TC><<<grid, W * 32, sm, s>>>(a, g0, g1 ? g1 : g0,
                                                        (const float2*)p->tw_l,
                                                        (const float2*)p->tw_n, (float2*)wfold,
                                                        rowmax);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}
template <int FF>
void launch_fwd(const sht_plan* p, const float* g0, const float* g1, int64_t planes, float* wfold,
                cudaStream_t s, float* rowmax) {
  constexpr int TLIN = (64 * FF) % 3 == 0 ? 64 * FF / 3 - 1 : -1;  // T + 1 = 2 nlon / 3
  if (TLIN >= 0 && p->T == TLIN)
    launch_fwd_t<FF, TLIN>(p, g0, g1, planes, wfold, s, rowmax);
  else
    launch_fwd_t<FF, -1>(p, g0, g1, planes, wfold, s, rowmax);
}

template <int FF, int NF>
void launch_inv_nf(const sht_plan* p, int mode, const float* wP, const float* wD, int64_t planes,
                   float* out0, float* out1, cudaStream_t s) {
  constexpr int NO = NF == 1 ? 1 : 2;
  FastUnfoldArgs a{p->nlat, p->nlon, p->T, p->H, p->nlat_odd ? 1 : 0, mode, kWarps / 2 / NO,
                   planes, (float)p->radius};
  dim3 grid((unsigned)div_up(planes, a.G), (unsigned)p->H);
  const size_t sm = sizeof(float2) * (kWarps * WarpSmem<FF>::kFloats2 + FF * 32);
  SHT_CUDA_OR_THROW(cudaFuncSetAttribute(fast_inverse_unfold<FF, NF>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  fast_inverse_unfold<FF, NF><<<grid, kWarps * 32, sm, s>>>(
      a, (const float2*)wP, (const float2*)(wD ? wD : wP), p->d_coslat, (const float2*)p->tw_l,
      (const float2*)p->tw_n, out0, out1 ? out1 : out0);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template <int FF>
void launch_inv(const sht_plan* p, int mode, const float* wP, const float* wD, int64_t planes,
                float* out0, float* out1, cudaStream_t s) {
  if (mode == kUnfoldWind)
    launch_inv_pair<FF, 4>(p, mode, wP, wD, planes, out0, out1, s);
  else if (mode == kUnfoldGradient && planes % 2 == 0)
    launch_inv_pair<FF, 2>(p, mode, wP, wD, planes, out0, out1, s);
  else if (mode == kUnfoldGradient)
    launch_inv_nf<FF, 2>(p, mode, wP, wD, planes, out0, out1, s);
  else if (planes % 2 == 0)
    launch_inv_pair<FF, 1>(p, mode, wP, wD, planes, out0, out1, s);
  else
    launch_inv_nf<FF, 1>(p, mode, wP, wD, planes, out0, out1, s);
}

}  // namespace

bool fast_fft_supported(const sht_plan* p) {
  if (p->prec == SHT_PREC_F64 || p->L % 32 != 0) return false;
  switch (p->L / 32) {
    case 2: case 3: case 4: case 6: case 8: case 12: case 16: case 24: return true;
    default: return false;
  }
}

void fast_fft_init_constants(cudaStream_t s) {
  float2 w24[24], w32[32], w16[16];
  for (int k = 0; k < 24; ++k) w24[k] = make_float2((float)cos(-2 * kPi * k / 24), (float)sin(-2 * kPi * k / 24));
  for (int k = 0; k < 32; ++k) w32[k] = make_float2((float)cos(-2 * kPi * k / 32), (float)sin(-2 * kPi * k / 32));
  for (int k = 0; k < 16; ++k) w16[k] = make_float2((float)cos(-2 * kPi * k / 16), (float)sin(-2 * kPi * k / 16));
  SHT_CUDA_OR_THROW(cudaMemcpyToSymbolAsync(c_w24, w24, sizeof(w24), 0, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaMemcpyToSymbolAsync(c_w32, w32, sizeof(w32), 0, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaMemcpyToSymbolAsync(c_w16, w16, sizeof(w16), 0, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
}

void fast_forward_fold(const sht_plan* p, const float* g0, const float* g1, int64_t planes,
                       float* wfold, cudaStream_t s, float* rowmax) {
  switch (p->L / 32) {
    case 2: launch_fwd<2>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 3: launch_fwd<3>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 4: launch_fwd<4>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 6: launch_fwd<6>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 8: launch_fwd<8>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 12: launch_fwd<12>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 16: launch_fwd<16>(p, g0, g1, planes, wfold, s, rowmax); break;
    case 24: launch_fwd<24>(p, g0, g1, planes, wfold, s, rowmax); break;
    default: throw Error{SHT_ERR_STATE, "fast FFT: unsupported length"};
  }
}

void fast_inverse_unfold(const sht_plan* p, int mode, const float* wP, const float* wD,
                         int64_t planes, float* out0, float* out1, cudaStream_t s) {
  switch (p->L / 32) {
    case 2: launch_inv<2>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 3: launch_inv<3>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 4: launch_inv<4>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 6: launch_inv<6>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 8: launch_inv<8>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 12: launch_inv<12>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 16: launch_inv<16>(p, mode, wP, wD, planes, out0, out1, s); break;
    case 24: launch_inv<24>(p, mode, wP, wD, planes, out0, out1, s); break;
    default: throw Error{SHT_ERR_STATE, "fast FFT: unsupported length"};
  }
}

}  // namespace sht
