// FP64 geometry on the GPU: Gauss-Legendre nodes and weights by Newton
// iteration, the normalised associated-Legendre recurrence and dP/dphi in the
// equator-folded (order, parity) layout, the Gram correction of the analysis
// rows, and the vector-analysis tables.  Everything here runs once per plan.
//
// Reference: src/arwen_global/spectral/grid.py:97-126 (leggauss nodes,
// ascending, weights summing to 2), legendre.py:76-146 (recurrence and
// derivative, operand order kept), transform.py:97-119 (Gram-solved analysis
// rows), vector.py:19-34 (rotation/shear weights).
#include "sht_plan.h"

namespace sht {
namespace {

// --------------------------------------------------------- Gauss nodes
// One thread per node pair: Newton on P_n from the asymptotic guess
// x0 = cos(pi (k + 3/4) / (n + 1/2)); P_n and P_n' by the three-term
// recurrence; w = 2 / ((1 - x^2) P_n'(x)^2).  Node k (largest first) is
// stored at mu[n-1-k] = +x and mu[k] = -x so the array ascends.
__global__ void gauss_newton_kernel(int n, double* mu, double* w) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int half = n / 2;
  if (k >= half) {
    if (k == half && (n & 1)) {  // the equator node of an odd grid
      // P_j(0) = -(j-1)/j P_{j-2}(0) from P_0 = 1, P_1 = 0; then
      // P_n'(0) = n (0 * P_n - P_{n-1}) / (0 - 1) = n P_{n-1}(0).
      double pm1 = 1.0, pj = 0.0;
      for (int j = 2; j <= n; ++j) {
        double pn = (-(double)(j - 1) * pm1) / (double)j;
        pm1 = pj;
        pj = pn;
      }
      double dp = (double)n * pm1;
      mu[half] = 0.0;
      w[half] = 2.0 / (dp * dp);
    }
    return;
  }
  double x = cos(kPi * ((double)k + 0.75) / ((double)n + 0.5));
  double dp = 1.0;
  for (int it = 0; it < 100; ++it) {
    double pm1 = 1.0, pj = x;
    for (int j = 2; j <= n; ++j) {
      double pn = ((double)(2 * j - 1) * x * pj - (double)(j - 1) * pm1) / (double)j;
      pm1 = pj;
      pj = pn;
    }
    dp = (double)n * (x * pj - pm1) / (x * x - 1.0);
    double dx = pj / dp;
    x -= dx;
    if (fabs(dx) <= 1e-16) break;
  }
  // Final derivative at the converged node for the weight.
  {
    double pm1 = 1.0, pj = x;
    for (int j = 2; j <= n; ++j) {
      double pn = ((double)(2 * j - 1) * x * pj - (double)(j - 1) * pm1) / (double)j;
      pm1 = pj;
      pj = pn;
    }
    dp = (double)n * (x * pj - pm1) / (x * x - 1.0);
  }
  double wk = 2.0 / ((1.0 - x * x) * dp * dp);
  mu[n - 1 - k] = x;
  mu[k] = -x;
  w[n - 1 - k] = wk;
  w[k] = wk;
}

// Scale the weights to sum to exactly 2 (as leggauss does) and form cos(phi).
__global__ void gauss_finish_kernel(int n, const double* mu, double* w, double* coslat) {
  __shared__ double part[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += w[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) part[threadIdx.x] += part[threadIdx.x + st];
    __syncthreads();
  }
  double scale = 2.0 / part[0];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    w[i] = w[i] * scale;
    double x = mu[i];
    coslat[i] = sqrt(fmax(0.0, 1.0 - x * x));
  }
}

// ------------------------------------------------ Legendre recurrence
struct TabGeom {
  int T, H, Hx;
  const int64_t* syn_off;  // [m*2+q]
};

// One thread per (m, h): the orthonormal recurrence at mu_h (southern node
// of pair h) for every n in [m, T], writing P and dP/dphi into the folded
// synthesis layout.  Products keep the reference's operand order and are
// not contracted into FMAs, so each value is the rounding of the same
// expression the reference evaluates.
__global__ void legendre_kernel(TabGeom g, const double* mu, double* P, double* dP) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  int m = blockIdx.y;
  if (h >= g.H) return;
  const double x = mu[h];
  const double root = __dsqrt_rn(fmax(0.0, __dsub_rn(1.0, __dmul_rn(x, x))));
  const double denom = __dsub_rn(__dmul_rn(x, x), 1.0);
  const double coslat = root;
  double diag = 1.0 / sqrt(4.0 * kPi);
  for (int k = 1; k <= m; ++k) {
    double c = __ddiv_rn((double)(2 * k + 1), __dmul_rn(2.0, (double)k));
    diag = __dmul_rn(__dmul_rn(-__dsqrt_rn(c), root), diag);
  }
  const int T = g.T;
  const int64_t o0 = g.syn_off[m * 2 + 0];
  const int64_t o1 = g.syn_off[m * 2 + 1];
  // n = m
  double p2 = 0.0, p1 = diag;
  {
    double d = 0.0;
    if (m >= 1) d = __ddiv_rn(__dmul_rn(coslat, __dmul_rn(__dmul_rn((double)m, x), diag)), denom);
    P[o0 + h] = diag;
    dP[o0 + h] = d;
  }
  for (int n = m + 1; n <= T; ++n) {
    double pn;
    if (n == m + 1) {
      pn = __dmul_rn(__dmul_rn(__dsqrt_rn((double)(2 * m + 3)), x), diag);
    } else {
      double nn = (double)n, mm = (double)m;
      double a = __dsqrt_rn(__ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn(4.0, nn), nn), 1.0),
                                      (double)((long long)n * n - (long long)m * m)));
      double n1 = nn - 1.0;
      double b = __dsqrt_rn(__ddiv_rn(__dsub_rn(__dmul_rn(n1, n1), __dmul_rn(mm, mm)),
                                      __dsub_rn(__dmul_rn(__dmul_rn(4.0, n1), n1), 1.0)));
      pn = __dmul_rn(a, __dsub_rn(__dmul_rn(x, p1), __dmul_rn(b, p2)));
    }
    // dP/dphi = coslat * (n x P_n - c P_{n-1}) / denom,
    // c = sqrt((n^2 - m^2)(2n+1)/(2n-1)).
    double nn = (double)n;
    double cc = __dsqrt_rn(__ddiv_rn(
        __dmul_rn((double)((long long)n * n - (long long)m * m), __dadd_rn(__dmul_rn(2.0, nn), 1.0)),
        __dsub_rn(__dmul_rn(2.0, nn), 1.0)));
    double num = __dsub_rn(__dmul_rn(__dmul_rn(nn, x), pn), __dmul_rn(cc, p1));
    double d = __ddiv_rn(__dmul_rn(coslat, num), denom);
    int q = (n - m) & 1;
    int i = (n - m) >> 1;
    int64_t off = (q ? o1 : o0) + (int64_t)i * g.Hx + h;
    P[off] = pn;
    dP[off] = d;
    p2 = p1;
    p1 = pn;
  }
}

// ------------------------------------------------------ Gram correction
// E = G - I per (m, q) block, G[i][i'] = sum_h c_h ((P[i][h] w_h) 2 pi) P[i'][h]
// with c_h = 2 for a latitude pair and 1 for the equator row of an odd grid.
struct GramArgs {
  int H, Hx, nlat_odd;
  const int64_t* syn_off;
  const int64_t* ana_off;
  const int64_t* e_off;  // E block offsets (e*e)
  const int* e;          // counts [m*2+q]
  const int* ex;         // padded counts
  const double* w;
};

constexpr int GT = 16;

__global__ void gram_e_kernel(GramArgs a, const double* P, double* E) {
  int pq = blockIdx.z;  // m*2+q
  int e = a.e[pq];
  int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
  if (i0 >= e || j0 >= e) return;
  const double* Pb = P + a.syn_off[pq];
  __shared__ double si[GT][GT + 1], sj[GT][GT + 1];
  int tx = threadIdx.x % GT, ty = threadIdx.x / GT;
  double acc = 0.0;
  for (int h0 = 0; h0 < a.H; h0 += GT) {
    int h = h0 + tx;
    int ri = i0 + ty, rj = j0 + ty;
    double wh = h < a.H ? a.w[h] : 0.0;
    double ch = (a.nlat_odd && h == a.H - 1) ? 1.0 : 2.0;
    si[ty][tx] = (ri < e && h < a.H) ? ch * ((Pb[(int64_t)ri * a.Hx + h] * wh) * (2.0 * kPi)) : 0.0;
    sj[ty][tx] = (rj < e && h < a.H) ? Pb[(int64_t)rj * a.Hx + h] : 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GT; ++k) acc += si[ty][k] * sj[tx][k];
    __syncthreads();
  }
  int i = i0 + ty, j = j0 + tx;
  if (i < e && j < e) E[a.e_off[pq] + (int64_t)i * e + j] = acc - (i == j ? 1.0 : 0.0);
}

// A[h][i] = rows[i][h] - sum_i' E[i][i'] rows[i'][h], rows = (P w) 2 pi,
// written in the analysis layout.  First-order Neumann solve of G A = rows:
// |E| is O(T eps), so the neglected E^2 term is far below float64 rounding.
__global__ void gram_apply_kernel(GramArgs a, const double* P, const double* E, double* A) {
  int pq = blockIdx.z;
  int e = a.e[pq];
  int i0 = blockIdx.y * GT, h0 = blockIdx.x * GT;
  if (i0 >= e || h0 >= a.H) return;
  const double* Pb = P + a.syn_off[pq];
  const double* Eb = E + a.e_off[pq];
  __shared__ double se[GT][GT + 1], sr[GT][GT + 1];
  int tx = threadIdx.x % GT, ty = threadIdx.x / GT;
  int i = i0 + ty, h = h0 + tx;
  double wh = h < a.H ? a.w[h] : 0.0;
  double acc = 0.0;
  for (int k0 = 0; k0 < e; k0 += GT) {
    int kk = k0 + tx;
    se[ty][tx] = (i < e && kk < e) ? Eb[(int64_t)i * e + kk] : 0.0;
    int kr = k0 + ty;
    sr[ty][tx] = (kr < e && h < a.H) ? (Pb[(int64_t)kr * a.Hx + h] * wh) * (2.0 * kPi) : 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < GT; ++k) acc += se[ty][k] * sr[k][tx];
    __syncthreads();
  }
  if (i < e && h < a.H) {
    double rows = (Pb[(int64_t)i * a.Hx + h] * wh) * (2.0 * kPi);
    A[a.ana_off[pq] + (int64_t)h * a.ex[pq] + i] = rows - acc;
  }
}

// Vector-analysis tables (vector.py:19-34): rot = ((w/cos) 2pi/a) P and
// shear = (w 2pi/a) dP, in the analysis layout.
__global__ void vector_tables_kernel(GramArgs a, double radius, const double* coslat,
                                     const double* P, const double* dP, double* R,
                                     double* S) {
  int pq = blockIdx.z;
  int e = a.e[pq];
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  int i = blockIdx.y;
  if (i >= e || h >= a.H) return;
  double scale = 2.0 * kPi / radius;
  int64_t src = a.syn_off[pq] + (int64_t)i * a.Hx + h;
  int64_t dst = a.ana_off[pq] + (int64_t)h * a.ex[pq] + i;
  R[dst] = ((a.w[h] / coslat[h]) * scale) * P[src];
  S[dst] = (a.w[h] * scale) * dP[src];
}

__global__ void cast_kernel(const double* in, float* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

template <typename T>
T* dalloc(int64_t n) {
  T* p = nullptr;
  SHT_CUDA_OR_THROW(cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)));
  return p;
}

}  // namespace

void build_geometry_and_tables(sht_plan* p, cudaStream_t s) {
  const int T = p->T;
  p->H = (p->nlat + 1) / 2;
  p->nlat_odd = (p->nlat & 1) != 0;
  p->Hx = (int)round_up(p->H, 4);
  p->L = p->nlon / 2;

  // Per (m, q) offsets.
  const int nb = 2 * (T + 1);
  p->e.assign(nb, 0);
  p->ex.assign(nb, 0);
  p->syn_off.assign(nb, 0);
  p->ana_off.assign(nb, 0);
  p->cf_row.assign(nb, 0);
  std::vector<int64_t> e_off(nb, 0);
  int64_t so = 0, ao = 0, cr = 0, eo = 0;
  for (int m = 0; m <= T; ++m)
    for (int q = 0; q < 2; ++q) {
      int idx = m * 2 + q;
      int e = parity_count(T, m, q);
      p->e[idx] = e;
      p->ex[idx] = (int)round_up(e, 4);
      p->syn_off[idx] = so;
      p->ana_off[idx] = ao;
      p->cf_row[idx] = cr;
      e_off[idx] = eo;
      so += (int64_t)e * p->Hx;
      ao += (int64_t)p->H * p->ex[idx];
      cr += e;
      eo += (int64_t)e * e;
    }
  p->syn_total = so;
  p->ana_total = ao;
  p->cf_rows = cr;

  // Geometry.
  p->d_mu = dalloc<double>(p->nlat);
  p->d_w = dalloc<double>(p->nlat);
  p->d_coslat = dalloc<double>(p->nlat);
  {
    int half = p->nlat / 2 + 1;
    gauss_newton_kernel<<<(half + 127) / 128, 128, 0, s>>>(p->nlat, p->d_mu, p->d_w);
    gauss_finish_kernel<<<1, 256, 0, s>>>(p->nlat, p->d_mu, p->d_w, p->d_coslat);
    SHT_CUDA_OR_THROW(cudaGetLastError());
  }

  if (p->geometry_only) {
    SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
    p->h_mu.resize(p->nlat);
    p->h_w.resize(p->nlat);
    p->h_coslat.resize(p->nlat);
    SHT_CUDA_OR_THROW(cudaMemcpy(p->h_mu.data(), p->d_mu, 8 * p->nlat, cudaMemcpyDeviceToHost));
    SHT_CUDA_OR_THROW(cudaMemcpy(p->h_w.data(), p->d_w, 8 * p->nlat, cudaMemcpyDeviceToHost));
    SHT_CUDA_OR_THROW(cudaMemcpy(p->h_coslat.data(), p->d_coslat, 8 * p->nlat,
                                 cudaMemcpyDeviceToHost));
    return;
  }

  // Device copies of the bookkeeping.
  int64_t* d_syn = dalloc<int64_t>(nb);
  int64_t* d_ana = dalloc<int64_t>(nb);
  int64_t* d_eoff = dalloc<int64_t>(nb);
  int* d_e = dalloc<int>(nb);
  int* d_ex = dalloc<int>(nb);
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(d_syn, p->syn_off.data(), 8 * nb, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(d_ana, p->ana_off.data(), 8 * nb, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(d_eoff, e_off.data(), 8 * nb, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(d_e, p->e.data(), 4 * nb, cudaMemcpyHostToDevice, s));
  SHT_CUDA_OR_THROW(cudaMemcpyAsync(d_ex, p->ex.data(), 4 * nb, cudaMemcpyHostToDevice, s));

  // FP64 master tables.
  double* P64 = dalloc<double>(p->syn_total);
  double* dP64 = dalloc<double>(p->syn_total);
  double* A64 = dalloc<double>(p->ana_total);
  double* R64 = dalloc<double>(p->ana_total);
  double* S64 = dalloc<double>(p->ana_total);
  double* E64 = dalloc<double>(eo);
  SHT_CUDA_OR_THROW(cudaMemsetAsync(P64, 0, 8 * std::max<int64_t>(p->syn_total, 1), s));
  SHT_CUDA_OR_THROW(cudaMemsetAsync(dP64, 0, 8 * std::max<int64_t>(p->syn_total, 1), s));
  SHT_CUDA_OR_THROW(cudaMemsetAsync(A64, 0, 8 * std::max<int64_t>(p->ana_total, 1), s));
  SHT_CUDA_OR_THROW(cudaMemsetAsync(R64, 0, 8 * std::max<int64_t>(p->ana_total, 1), s));
  SHT_CUDA_OR_THROW(cudaMemsetAsync(S64, 0, 8 * std::max<int64_t>(p->ana_total, 1), s));

  TabGeom g{T, p->H, p->Hx, d_syn};
  legendre_kernel<<<dim3((p->H + 127) / 128, T + 1), 128, 0, s>>>(g, p->d_mu, P64, dP64);
  SHT_CUDA_OR_THROW(cudaGetLastError());

  GramArgs ga{p->H, p->Hx, p->nlat_odd ? 1 : 0, d_syn, d_ana, d_eoff, d_e, d_ex, p->d_w};
  int emax = parity_count(T, 0, 0);
  dim3 ge((unsigned)div_up(emax, GT), (unsigned)div_up(emax, GT), (unsigned)nb);
  gram_e_kernel<<<ge, GT * GT, 0, s>>>(ga, P64, E64);
  dim3 gap((unsigned)div_up(p->H, GT), (unsigned)div_up(emax, GT), (unsigned)nb);
  gram_apply_kernel<<<gap, GT * GT, 0, s>>>(ga, P64, E64, A64);
  vector_tables_kernel<<<dim3((unsigned)div_up(p->H, 128), (unsigned)emax, (unsigned)nb), 128, 0, s>>>(
      ga, p->radius, p->d_coslat, P64, dP64, R64, S64);
  SHT_CUDA_OR_THROW(cudaGetLastError());

  if (p->prec == SHT_PREC_F64) {
    p->basis = P64;
    p->dbasis = dP64;
    p->analysis = A64;
    p->rot = R64;
    p->shear = S64;
  } else {
    float* tabs[5];
    const double* src[5] = {P64, dP64, A64, R64, S64};
    int64_t sz[5] = {p->syn_total, p->syn_total, p->ana_total, p->ana_total, p->ana_total};
    for (int t = 0; t < 5; ++t) {
      tabs[t] = dalloc<float>(sz[t]);
      cast_kernel<<<592, 256, 0, s>>>(src[t], tabs[t], sz[t]);
    }
    SHT_CUDA_OR_THROW(cudaGetLastError());
    p->basis = tabs[0];
    p->dbasis = tabs[1];
    p->analysis = tabs[2];
    p->rot = tabs[3];
    p->shear = tabs[4];
    if (p->prec == SHT_PREC_SPLIT16) build_tc_tables(p, P64, dP64, A64, R64, S64, s);
    SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
    for (int t = 0; t < 5; ++t) cudaFree((void*)src[t]);
  }
  SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
  cudaFree(E64);
  cudaFree(d_syn);
  cudaFree(d_ana);
  cudaFree(d_eoff);
  cudaFree(d_e);
  cudaFree(d_ex);

  p->h_mu.resize(p->nlat);
  p->h_w.resize(p->nlat);
  p->h_coslat.resize(p->nlat);
  SHT_CUDA_OR_THROW(cudaMemcpy(p->h_mu.data(), p->d_mu, 8 * p->nlat, cudaMemcpyDeviceToHost));
  SHT_CUDA_OR_THROW(cudaMemcpy(p->h_w.data(), p->d_w, 8 * p->nlat, cudaMemcpyDeviceToHost));
  SHT_CUDA_OR_THROW(cudaMemcpy(p->h_coslat.data(), p->d_coslat, 8 * p->nlat, cudaMemcpyDeviceToHost));
}

}  // namespace sht
