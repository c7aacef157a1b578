// Per-degree semi-implicit maps in the vertical-mode basis.
//
// VerticalModeSemiImplicit (src/arwen_global/semi_implicit.py:845-953) with
// x = (theta, ln ps), k_n^2 = n(n+1)/a^2, the structure M = -B C = V L V^-1
// and the thermodynamic block C B = W Mu W^-1:
//
//   solve_shifted (kSolve, 921-953):
//     forcing = D + tau k^2 (B x)
//     D'      = V diag(1/(1 + tau^2 k^2 lambda)) V^-1 forcing
//     x'      = x + tau C D'
//   apply, off-centred Crank-Nicolson with weight alpha (kApply, 887-919):
//     forcing = D + dt k^2 B x - alpha (1-alpha) dt^2 k^2 M D
//             = D + dt k^2 B (x + alpha (1-alpha) dt C D)
//     D'      = V diag(1/(1 + (alpha dt)^2 k^2 lambda)) V^-1 forcing
//     x'      = x + dt C ((1-alpha) D + alpha D')
//   linear_tendencies, the weighted linear operator itself (kLinear, 796-813):
//     D_t = w k^2 (B x),   x_t = w (C D)
//     (projected like the maps, without the degree-zero pass-through: the
//     tendency of degree zero is w k_0^2 B x = 0 for D and w C D for x)
//   half_apply, the square root of that map (kHalf, 845-877 with
//   symmetric_half_maps, 611-663):
//     D' = V [diag(p_D) V^-1 D + diag(q_D) V^-1 (k^2 B x)]
//     x' = W [diag(p_x) W^-1 x + diag(q_x) W^-1 (C D)]
//     p + i q omega = sqrt((1 + i (1-alpha) omega dt) / (1 - i alpha omega dt))
//     per mode frequency omega = k sqrt(lambda_j) (D block) or
//     k sqrt(-mu_j) (x block), principal root; omega = 0 gives p = 1, q = dt/2.
// Degree zero passes through and the outputs are projected (_finish,
// semi_implicit.py:815-843).  The per-degree inverses are applied modally
// (helmholtz_inverse, semi_implicit.py:585-609) instead of as a stored
// (T+1, nlev, nlev) stack: a few small mat-vecs per coefficient, with the
// operators held in shared memory by persistent CTAs and each thread
// accumulating six matrix rows against one 32-order column block.
//
// Optional outputs: `metric` (the reference's max |D' - D|, through an
// atomicMax on the value's bits, which orders like the value for numbers
// >= 0), and `cfold` (D' written straight into the folded synthesis operand
// of the plan, rows (m, q, i) with the levels as planes, plus the row
// maxima of the split-precision path): the Helmholtz solve as the prologue
// of the divergence synthesis, without a pack pass.
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

// The half-map scalars of one mode: p + i q omega = sqrt(g), with
// g = (1 + i (1-a) y) / (1 - i a y) = (1 - a (1-a) y^2 + i y) / (1 + a^2 y^2),
// y = omega dt; principal square root by the half-angle formulas, the
// cancelling branch avoided (Re g >= 0: re = sqrt((|g| + Re g) / 2),
// im = Im g / (2 re); otherwise im first).
__device__ __forceinline__ void half_map_scalars(double omega, double dt, double alpha,
                                                 double& p, double& q) {
  if (!(omega > 0.0)) {
    p = 1.0;
    q = 0.5 * dt;
    return;
  }
  const double y = omega * dt;
  const double den = 1.0 + alpha * alpha * y * y;
  const double a = (1.0 - alpha * (1.0 - alpha) * y * y) / den;
  const double b = y / den;
  const double r = hypot(a, b);
  double re, im;
  if (a >= 0.0) {
    re = sqrt(0.5 * (r + a));
    im = b / (2.0 * re);
  } else {
    im = copysign(sqrt(0.5 * (r - a)), b);
    re = b / (2.0 * im);
  }
  p = re;
  q = im / omega;
}

struct SemiArgs {
  int Tn, nlev, mode;
  double radius, dt, alpha;
  int64_t cf_planes;  // Cfold column count (the levels), when cfold is set
};

// Shared-memory plan of one mode (element counts in T).
struct SmemPlan {
  int ldB, ldC, ldV, ldW, vp;
  int oB, oC, oV, oVi, oLam, oW, oWi, oMu, oPQ, nmat;  // matrix offsets (T elements)
  int nvec;                                               // vectors of [vp][32] V2<T>
};

__host__ __device__ inline SmemPlan smem_plan(int nlev, int mode) {
  SmemPlan s{};
  const int L1 = nlev + 1;
  s.ldB = padded(L1);
  s.ldC = padded(nlev);
  s.ldV = padded(nlev);
  s.ldW = padded(L1);
  s.vp = padded(L1);
  s.oB = 0;
  s.oC = s.oB + padded_rows(nlev) * s.ldB;
  s.oV = s.oC + padded_rows(L1) * s.ldC;
  s.oVi = s.oV + padded_rows(nlev) * s.ldV;
  s.oLam = s.oVi + padded_rows(nlev) * s.ldV;
  s.oW = s.oLam + padded(nlev);
  const bool half = mode == kSemiHalf;
  s.oWi = s.oW + (half ? padded_rows(L1) * s.ldW : 0);
  s.oMu = s.oWi + (half ? padded_rows(L1) * s.ldW : 0);
  s.oPQ = s.oMu + (half ? padded(L1) : 0);
  // p_D, q_D (nlev each) and p_x, q_x (nlev + 1 each) of the current degree
  s.nmat = s.oPQ + (half ? 2 * padded(nlev) + 2 * padded(L1) : 0);
  s.nmat = (s.nmat + 1) & ~1;  // the V2<T> vectors that follow stay aligned
  s.nvec = half ? 5 : 4;
  return s;
}

// Persistent: each CTA copies the operators into shared memory once (rows
// padded to multiples of 4 with zeros) and then walks items (degree n, 32
// consecutive orders), n fastest so that CTAs running together read
// neighbouring coefficient rows.  Items wholly above the triangle write zeros.
template <typename T>
__global__ void __launch_bounds__(256) semi_implicit_kernel(
    SemiArgs a, const T* __restrict__ mats, const V2<T>* __restrict__ div,
    const V2<T>* __restrict__ theta, const V2<T>* __restrict__ lnps, V2<T>* __restrict__ odiv,
    V2<T>* __restrict__ otheta, V2<T>* __restrict__ olnps, T* __restrict__ metric,
    V2<T>* __restrict__ cfold, float* __restrict__ rowmax) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Tn = a.Tn, nlev = a.nlev, mode = a.mode;
  const int L1 = nlev + 1;
  const SmemPlan sp = smem_plan(nlev, mode);
  T* sm = reinterpret_cast<T*>(smem_raw);
  T* sB = sm + sp.oB;    // nlev x L1
  T* sC = sm + sp.oC;    // L1 x nlev
  T* sV = sm + sp.oV;    // nlev x nlev
  T* sVi = sm + sp.oVi;  // nlev x nlev
  T* sLam = sm + sp.oLam;
  T* sW = sm + sp.oW;    // L1 x L1 (kSemiHalf)
  T* sWi = sm + sp.oWi;
  T* sMu = sm + sp.oMu;
  T* sPQ = sm + sp.oPQ;  // p_D, q_D, p_x, q_x of the current degree
  V2<T>* xs = reinterpret_cast<V2<T>*>(sm + sp.nmat);  // [vp][32] each
  V2<T>* fs = xs + sp.vp * 32;
  V2<T>* gs = fs + sp.vp * 32;
  V2<T>* ds = gs + sp.vp * 32;
  V2<T>* hs = ds + sp.vp * 32;  // kSemiHalf only
  __shared__ float s_rowmax[2 * kMaxLev];
  __shared__ T s_metric[8];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  {
    const T* B = mats;              // nlev x (nlev+1)
    const T* C = B + nlev * L1;     // (nlev+1) x nlev
    const T* V = C + L1 * nlev;     // nlev x nlev
    const T* Vi = V + nlev * nlev;  // nlev x nlev
    const T* lam = Vi + nlev * nlev;
    const T* W = lam + nlev;        // (nlev+1) x (nlev+1), when present
    const T* Wi = W + L1 * L1;
    const T* mu = Wi + L1 * L1;
    for (int e = tid; e < padded_rows(nlev) * sp.ldB; e += 256) {
      const int i = e / sp.ldB, j = e - i * sp.ldB;
      sB[e] = (i < nlev && j < L1) ? B[i * L1 + j] : T(0);
    }
    for (int e = tid; e < padded_rows(L1) * sp.ldC; e += 256) {
      const int i = e / sp.ldC, j = e - i * sp.ldC;
      sC[e] = (i < L1 && j < nlev) ? C[i * nlev + j] : T(0);
    }
    for (int e = tid; e < padded_rows(nlev) * sp.ldV; e += 256) {
      const int i = e / sp.ldV, j = e - i * sp.ldV;
      const bool in = i < nlev && j < nlev;
      sV[e] = in ? V[i * nlev + j] : T(0);
      sVi[e] = in ? Vi[i * nlev + j] : T(0);
    }
    for (int e = tid; e < padded(nlev); e += 256) sLam[e] = e < nlev ? lam[e] : T(0);
    if (mode == kSemiHalf) {
      for (int e = tid; e < padded_rows(L1) * sp.ldW; e += 256) {
        const int i = e / sp.ldW, j = e - i * sp.ldW;
        const bool in = i < L1 && j < L1;
        sW[e] = in ? W[i * L1 + j] : T(0);
        sWi[e] = in ? Wi[i * L1 + j] : T(0);
      }
      for (int e = tid; e < padded(L1); e += 256) sMu[e] = e < L1 ? mu[e] : T(0);
    }
    // Vector padding rows stay zero for the whole launch.
    for (int e = tid; e < sp.nvec * sp.vp * 32; e += 256) xs[e] = mk2<T>(T(0), T(0));
    for (int e = tid; e < 2 * kMaxLev; e += 256) s_rowmax[e] = 0.f;
    if (tid < 8) s_metric[tid] = T(0);
  }
  const int64_t t1 = Tn + 1;
  const int64_t lev = t1 * t1;  // one level of coefficients
  const int nmb = (Tn + 1 + 31) / 32;
  const T dt = T(a.dt), alpha = T(a.alpha);
  const bool off_centred = mode == kSemiApply && a.alpha != 1.0;
  T my_metric = T(0);
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
      if (i < nlev) ds[i * 32 + tx] = live ? div[i * lev + cidx] : mk2<T>(T(0), T(0));
    }
    const double k2d = (double)n * ((double)n + 1.0) / (a.radius * a.radius);
    const T k2 = T(k2d);
    if (mode == kSemiHalf) {
      // This degree's half-map scalars, once per item.
      const double k = sqrt(k2d);
      for (int j = tid; j < nlev; j += 256) {
        double p, q;
        half_map_scalars(k * sqrt((double)sLam[j]), a.dt, a.alpha, p, q);
        sPQ[j] = T(p);
        sPQ[padded(nlev) + j] = T(q);
      }
      for (int j = tid; j < L1; j += 256) {
        double p, q;
        half_map_scalars(k * sqrt(fmax(-(double)sMu[j], 0.0)), a.dt, a.alpha, p, q);
        sPQ[2 * padded(nlev) + j] = T(p);
        sPQ[2 * padded(nlev) + padded(L1) + j] = T(q);
      }
    }
    __syncthreads();
    // d_new written for row i of column tx: degree zero passes through, the
    // triangle projection, the metric and the fused synthesis operand.
    auto store_div = [&](int i, V2<T> dn) {
      const V2<T> d0 = ds[i * 32 + tx];
      if (n == 0) dn = d0;  // degree zero passes through
      if (m == 0) dn.y = T(0);
      if (!live) dn = mk2<T>(T(0), T(0));
      if (live) {
        const T ex = dn.x - d0.x, ey = dn.y - d0.y;
        my_metric = fmax(my_metric, sqrt(ex * ex + ey * ey));
      }
      if (m <= Tn) odiv[i * lev + cidx] = dn;
      if (cfold != nullptr && live) {
        const int q = (n - m) & 1, ii = (n - m) >> 1;
        const int64_t row = (int64_t)m * (Tn + 1) - (int64_t)m * (m - 1) / 2 +
                            (q ? parity_count(Tn, m, 0) : 0) + ii;
        cfold[row * a.cf_planes + i] = dn;
      }
      return dn;
    };
    auto store_x = [&](int i, V2<T> xn) {
      const V2<T> x = xs[i * 32 + tx];
      if (n == 0) xn = x;
      if (m == 0) xn.y = T(0);
      if (!live) xn = mk2<T>(T(0), T(0));
      if (m <= Tn) {
        if (i < nlev)
          otheta[i * lev + cidx] = xn;
        else
          olnps[cidx] = xn;
      }
    };
    // Row maxima of the fused synthesis operand: warp maxima over the 32
    // orders of this row, merged per CTA in shared memory.
    auto merge_rowmax = [&](int i, V2<T> dn) {
      if (rowmax == nullptr) return;
      float mre = live ? (float)fabs(dn.x) : 0.f, mim = live ? (float)fabs(dn.y) : 0.f;
      for (int off = 16; off > 0; off >>= 1) {
        mre = fmaxf(mre, __shfl_xor_sync(0xffffffffu, mre, off));
        mim = fmaxf(mim, __shfl_xor_sync(0xffffffffu, mim, off));
      }
      if (tx == 0) {
        atomicMax(reinterpret_cast<int*>(&s_rowmax[2 * i]), __float_as_int(mre));
        atomicMax(reinterpret_cast<int*>(&s_rowmax[2 * i + 1]), __float_as_int(mim));
      }
    };
    if (mode == kSemiHalf) {
      // fs = k^2 B x
      matvec<T>(sB, nlev, L1, xs, tx, ty, [&](int i, T ar, T ai) {
        fs[i * 32 + tx] = mk2<T>(k2 * ar, k2 * ai);
      });
      // hs = C D
      matvec<T>(sC, L1, nlev, ds, tx, ty, [&](int i, T ar, T ai) {
        hs[i * 32 + tx] = mk2<T>(ar, ai);
      });
      __syncthreads();
      const T* pD = sPQ;
      const T* qD = sPQ + padded(nlev);
      const T* pX = sPQ + 2 * padded(nlev);
      const T* qX = pX + padded(L1);
      // gs = diag(p_D) V^-1 D + diag(q_D) V^-1 fs
      matvec<T>(sVi, nlev, nlev, ds, tx, ty, [&](int i, T ar, T ai) {
        gs[i * 32 + tx] = mk2<T>(pD[i] * ar, pD[i] * ai);
      });
      __syncthreads();
      matvec<T>(sVi, nlev, nlev, fs, tx, ty, [&](int i, T ar, T ai) {
        const V2<T> g = gs[i * 32 + tx];
        gs[i * 32 + tx] = mk2<T>(g.x + qD[i] * ar, g.y + qD[i] * ai);
      });
      __syncthreads();
      // fs = diag(p_x) W^-1 x, then + diag(q_x) W^-1 hs (fs's k^2 B x is consumed)
      matvec<T>(sWi, L1, L1, xs, tx, ty, [&](int i, T ar, T ai) {
        fs[i * 32 + tx] = mk2<T>(pX[i] * ar, pX[i] * ai);
      });
      __syncthreads();
      matvec<T>(sWi, L1, L1, hs, tx, ty, [&](int i, T ar, T ai) {
        const V2<T> f = fs[i * 32 + tx];
        fs[i * 32 + tx] = mk2<T>(f.x + qX[i] * ar, f.y + qX[i] * ai);
      });
      __syncthreads();
      // D' = V gs, x' = W fs
      matvec<T>(sV, nlev, nlev, gs, tx, ty, [&](int i, T ar, T ai) {
        merge_rowmax(i, store_div(i, mk2<T>(ar, ai)));
      });
      matvec<T>(sW, L1, L1, fs, tx, ty, [&](int i, T ar, T ai) {
        store_x(i, mk2<T>(ar, ai));
      });
      continue;
    }
    if (mode == kSemiLinear) {
      // dt carries the weight w; the outputs are projected only.
      const T wk2 = dt * k2;
      matvec<T>(sB, nlev, L1, xs, tx, ty, [&](int i, T ar, T ai) {
        V2<T> v = mk2<T>(wk2 * ar, wk2 * ai);
        if (m == 0) v.y = T(0);
        if (!live) v = mk2<T>(T(0), T(0));
        if (m <= Tn) odiv[i * lev + cidx] = v;
      });
      matvec<T>(sC, L1, nlev, ds, tx, ty, [&](int i, T ar, T ai) {
        V2<T> v = mk2<T>(dt * ar, dt * ai);
        if (m == 0) v.y = T(0);
        if (!live) v = mk2<T>(T(0), T(0));
        if (m <= Tn) {
          if (i < nlev)
            otheta[i * lev + cidx] = v;
          else
            olnps[cidx] = v;
        }
      });
      continue;
    }
    const V2<T>* bx = xs;
    if (off_centred) {
      // gs = x + alpha (1-alpha) dt C D: the M D term folded into the B product
      const T c = alpha * (T(1) - alpha) * dt;
      matvec<T>(sC, L1, nlev, ds, tx, ty, [&](int i, T ar, T ai) {
        const V2<T> x = xs[i * 32 + tx];
        gs[i * 32 + tx] = mk2<T>(x.x + c * ar, x.y + c * ai);
      });
      __syncthreads();
      bx = gs;
    }
    // forcing = D + dt k2 (B bx)
    matvec<T>(sB, nlev, L1, bx, tx, ty, [&](int i, T ar, T ai) {
      const V2<T> d = ds[i * 32 + tx];
      fs[i * 32 + tx] = mk2<T>(d.x + dt * k2 * ar, d.y + dt * k2 * ai);
    });
    __syncthreads();
    // g = diag(1/(1 + (alpha dt)^2 k2 lambda)) V^-1 forcing
    const T adt = mode == kSemiApply ? alpha * dt : dt;
    matvec<T>(sVi, nlev, nlev, fs, tx, ty, [&](int i, T ar, T ai) {
      const T modal = T(1) / (T(1) + (adt * adt * k2) * sLam[i]);
      gs[i * 32 + tx] = mk2<T>(ar * modal, ai * modal);
    });
    __syncthreads();
    // D' = V g (into fs: the vector C multiplies next)
    matvec<T>(sV, nlev, nlev, gs, tx, ty, [&](int i, T ar, T ai) {
      const V2<T> dn = store_div(i, mk2<T>(ar, ai));
      merge_rowmax(i, dn);
      if (off_centred) {
        const V2<T> d = ds[i * 32 + tx];
        fs[i * 32 + tx] = mk2<T>((T(1) - alpha) * d.x + alpha * dn.x,
                                 (T(1) - alpha) * d.y + alpha * dn.y);
      } else {
        fs[i * 32 + tx] = dn;
      }
    });
    __syncthreads();
    // x' = x + dt C fs
    matvec<T>(sC, L1, nlev, fs, tx, ty, [&](int i, T ar, T ai) {
      const V2<T> x = xs[i * 32 + tx];
      store_x(i, mk2<T>(x.x + dt * ar, x.y + dt * ai));
    });
  }
  // CTA totals: one atomic per row maximum and one for the metric.
  if (rowmax != nullptr || metric != nullptr) {
    for (int off = 16; off > 0; off >>= 1) my_metric = fmax(my_metric, __shfl_xor_sync(0xffffffffu, my_metric, off));
    __syncthreads();
    if (tx == 0) s_metric[ty] = my_metric;
    __syncthreads();
    if (metric != nullptr && tid == 0) {
      T mx = T(0);
      for (int k = 0; k < 8; ++k) mx = fmax(mx, s_metric[k]);
      if constexpr (sizeof(T) == 8)
        atomicMax(reinterpret_cast<unsigned long long*>(metric),
                  (unsigned long long)__double_as_longlong(mx));
      else
        atomicMax(reinterpret_cast<unsigned*>(metric), __float_as_uint(mx));
    }
    if (rowmax != nullptr)
      for (int e = tid; e < 2 * nlev; e += 256)
        atomicMax(reinterpret_cast<int*>(rowmax + e), __float_as_int(s_rowmax[e]));
  }
}

}  // namespace

template <typename T>
void launch_semi_implicit(const sht_plan* p, int nlev, const T* mats, bool has_thermo, int mode,
                          double dt, double alpha, const T* div, const T* theta, const T* lnps,
                          T* odiv, T* otheta, T* olnps, T* metric, T* cfold, float* rowmax,
                          cudaStream_t s) {
  SHT_REQUIRE(nlev >= 1 && nlev <= kMaxLev, "nlev must be in [1, 96]");
  SHT_REQUIRE(mode == kSemiSolve || mode == kSemiApply || mode == kSemiHalf ||
                  mode == kSemiLinear,
              "unknown semi-implicit mode");
  SHT_REQUIRE(mode != kSemiHalf || has_thermo,
              "half_apply needs the thermodynamic block's modes (sht_vertical_create_modes)");
  const SmemPlan sp = smem_plan(nlev, mode);
  const size_t sm = sizeof(T) * (size_t)sp.nmat + sizeof(V2<T>) * 32 * (size_t)(sp.nvec * sp.vp);
  SHT_CUDA_OR_THROW(cudaFuncSetAttribute(semi_implicit_kernel<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int per_sm = 0, dev = 0, sms = 0;
  SHT_CUDA_OR_THROW(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, semi_implicit_kernel<T>, 256, sm));
  SHT_REQUIRE(per_sm > 0, "semi-implicit kernel does not fit on an SM at this nlev");
  SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
  SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int64_t items = div_up(p->T + 1, 32) * (int64_t)(p->T + 1);
  const int ctas = (int)std::min<int64_t>(items, (int64_t)per_sm * sms);
  SemiArgs a{p->T, nlev, mode, p->radius, dt, alpha, (int64_t)nlev};
  semi_implicit_kernel<T><<<ctas, dim3(32, 8), sm, s>>>(
      a, mats, (const V2<T>*)div, (const V2<T>*)theta, (const V2<T>*)lnps, (V2<T>*)odiv,
      (V2<T>*)otheta, (V2<T>*)olnps, metric, (V2<T>*)cfold, rowmax);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template <typename T>
void launch_helmholtz(const sht_plan* p, int nlev, const T* mats, double tau_w, const T* div,
                      const T* theta, const T* lnps, T* odiv, T* otheta, T* olnps,
                      cudaStream_t s) {
  launch_semi_implicit<T>(p, nlev, mats, false, kSemiSolve, tau_w, 1.0, div, theta, lnps, odiv,
                          otheta, olnps, nullptr, nullptr, nullptr, s);
}

#define INST(T)                                                                               \
  template void launch_semi_implicit<T>(const sht_plan*, int, const T*, bool, int, double,   \
                                        double, const T*, const T*, const T*, T*, T*, T*, T*, \
                                        T*, float*, cudaStream_t);                            \
  template void launch_helmholtz<T>(const sht_plan*, int, const T*, double, const T*,        \
                                    const T*, const T*, T*, T*, T*, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace sht
