// Plain SIMT Legendre contraction (the FP32 FFMA path and the FP64 parity
// path): for every (order m, degree parity q) block, C[x][r] = sum_k
// Tab[k][x] * D[k][r], with the plane/component rows r innermost in both the
// data and the output.  One launch covers the whole triangle: the work list
// holds (block, x-tile) items sorted by descending cost, so the large low-m
// blocks start first and the ragged high-m tail fills in behind them.  This
// replaces the reference's per-band dense strided-batched GEMMs
// (transform.py:1178-1274), which multiply the zeros above the triangle too.
#include <algorithm>
#include <type_traits>

#include "sht_plan.h"

namespace sht {
namespace {

// Tile shapes (x columns of the table x r data rows per CTA).  FP32 has two,
// chosen at run time (SHT_TUNE_SIMT_TILE): 128 x 128, and 64 x 128, whose
// narrower column tiles waste less on the ragged analysis blocks (X = the
// degrees of one order and parity) at the price of more table loads.
template <typename T, bool NARROW> struct SimtCfg;
template <> struct SimtCfg<float, false> {
  static constexpr int BX = 128, BR = 128, BK = 8, TMX = 8, TMR = 8, VW = 4;
  using V = float4;
};
template <> struct SimtCfg<float, true> {
  static constexpr int BX = 64, BR = 128, BK = 8, TMX = 4, TMR = 8, VW = 4;
  using V = float4;
};
template <> struct SimtCfg<double, false> {
  static constexpr int BX = 64, BR = 64, BK = 8, TMX = 4, TMR = 4, VW = 2;
  using V = double2;
};

template <typename T, bool NARROW>
__global__ void __launch_bounds__(256, 2) gemm_simt_kernel(const ShtGemmDesc* __restrict__ descs,
                                                        const ShtGemmItem* __restrict__ items,
                                                        const T* __restrict__ table,
                                                        const T* __restrict__ data,
                                                        T* __restrict__ out, int64_t R) {
  using C = SimtCfg<T, NARROW>;
  constexpr int BX = C::BX, BR = C::BR, BK = C::BK, TMX = C::TMX, TMR = C::TMR, VW = C::VW;
  constexpr int NTX = BX / TMX, NTR = BR / TMR;  // 16 x 16 threads
  constexpr int GX = TMX / VW, GR = TMR / VW;     // vector groups per thread
  static_assert(NTX * NTR == 256, "256 threads");

  const ShtGemmItem it = items[blockIdx.x];
  const ShtGemmDesc d = descs[it.problem];
  const int x0 = it.x0;
  const int64_t r0 = (int64_t)blockIdx.y * BR;
  const T* __restrict__ Tb = table + d.t_off;
  const T* __restrict__ Db = data + d.d_row * R;
  T* __restrict__ Cb = out + d.c_row * R;

  __shared__ __align__(16) T As[2][BK][BX];
  __shared__ __align__(16) T Bs[2][BK][BR];

  const int tid = threadIdx.x;
  // Thread -> a TMX x TMR block of contiguous x and r.  Warp w covers the
  // rows wr * BR/4 .. +BR/4 (wr = w % 4) and the columns wx * BX/2 .. +BX/2
  // (wx = w / 4); lane -> (lr = lane % 4, lx = lane / 4) within it.  A warp
  // whose rows or columns lie wholly past the problem's extent (the ragged x
  // tail of an analysis block, the last partial row block) skips its FFMAs:
  // the issue slots go to the other warps and CTAs of the SM.
  const int warp = tid >> 5, lane = tid & 31;
  const int r_base = (warp & 3) * (BR / 4) + (lane & 3) * TMR;
  const int x_base = (warp >> 2) * (BX / 2) + (lane >> 2) * TMX;
  static_assert(4 * TMR * 4 == BR && 8 * TMX * 2 == BX, "warp tiling covers the block");
  const bool busy = x0 + (warp >> 2) * (BX / 2) < d.X && r0 + (warp & 3) * (BR / 4) < R;

  // Global-load mapping: each tile is BK x B{X,R} = 8 x 128 (or 8 x 64);
  // thread loads LPT consecutive elements of one k-row.
  constexpr int LPT_A = BK * BX / 256, LPT_B = BK * BR / 256;
  const int la_k = tid / (BX / LPT_A), la_x = (tid % (BX / LPT_A)) * LPT_A;
  const int lb_k = tid / (BR / LPT_B), lb_r = (tid % (BR / LPT_B)) * LPT_B;

  T ra[LPT_A], rb[LPT_B];
  auto load_global = [&](int k0) {
    int k = k0 + la_k;
#pragma unroll
    for (int i = 0; i < LPT_A; ++i) {
      int x = x0 + la_x + i;
      ra[i] = (k < d.K && x < d.X) ? Tb[(int64_t)k * d.ldt + x] : T(0);
    }
    k = k0 + lb_k;
#pragma unroll
    for (int i = 0; i < LPT_B; ++i) {
      int64_t r = r0 + lb_r + i;
      rb[i] = (k < d.K && r < R) ? Db[(int64_t)k * R + r] : T(0);
    }
  };
  auto store_shared = [&](int buf) {
#pragma unroll
    for (int i = 0; i < LPT_A; ++i) As[buf][la_k][la_x + i] = ra[i];
#pragma unroll
    for (int i = 0; i < LPT_B; ++i) Bs[buf][lb_k][lb_r + i] = rb[i];
  };

  T acc[TMX][TMR];
#pragma unroll
  for (int i = 0; i < TMX; ++i)
#pragma unroll
    for (int j = 0; j < TMR; ++j) acc[i][j] = T(0);

  const int nk = (d.K + BK - 1) / BK;
  load_global(0);
  store_shared(0);
  __syncthreads();
  for (int kt = 0; kt < nk; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < nk) load_global((kt + 1) * BK);
    if (busy) {
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        T a[TMX], b[TMR];
#pragma unroll
        for (int g = 0; g < GX; ++g) {
          typename C::V v = *reinterpret_cast<const typename C::V*>(&As[buf][kk][x_base + g * VW]);
          const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
          for (int u = 0; u < VW; ++u) a[g * VW + u] = pv[u];
        }
#pragma unroll
        for (int g = 0; g < GR; ++g) {
          typename C::V v = *reinterpret_cast<const typename C::V*>(&Bs[buf][kk][r_base + g * VW]);
          const T* pv = reinterpret_cast<const T*>(&v);
#pragma unroll
          for (int u = 0; u < VW; ++u) b[g * VW + u] = pv[u];
        }
#pragma unroll
        for (int i = 0; i < TMX; ++i)
#pragma unroll
          for (int j = 0; j < TMR; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
    }
    if (kt + 1 < nk) {
      store_shared(buf ^ 1);
    }
    __syncthreads();
  }

  // Epilogue: C[x][r], r innermost.
#pragma unroll
  for (int i = 0; i < TMX; ++i) {
      int x = x0 + x_base + i;
      if (x >= d.X) continue;
      T* crow = Cb + (int64_t)x * R;
#pragma unroll
      for (int gr = 0; gr < GR; ++gr) {
        int64_t r = r0 + r_base + gr * VW;
        const T* av = &acc[i][gr * VW];
        if (r + VW <= R && (R % VW) == 0) {
          typename C::V v;
          T* pv = reinterpret_cast<T*>(&v);
#pragma unroll
          for (int w = 0; w < VW; ++w) pv[w] = av[w];
          *reinterpret_cast<typename C::V*>(crow + r) = v;
        } else {
#pragma unroll
          for (int w = 0; w < VW; ++w)
            if (r + w < R) crow[r + w] = av[w];
        }
      }
    }
}

}  // namespace

void build_gemm_items(sht_plan* p) {
  const int T = p->T;
  const int bx = p->prec == SHT_PREC_F64 ? SimtCfg<double, false>::BX : SimtCfg<float, false>::BX;
  p->gemm_bx = bx;
  // Every (m, q) is a problem, including the empty parity-1 block of m = T:
  // its synthesis item has K = 0 and writes the zeros the inverse FFT reads
  // from that waist slot (nothing else writes it).  Empty analysis blocks
  // have X = 0 and produce no items.
  std::vector<int> probs;
  for (int m = 0; m <= T; ++m)
    for (int q = 0; q < 2; ++q) probs.push_back(m * 2 + q);
  p->n_problems = (int)probs.size();
  for (int f = 0; f < 2; ++f) {
    auto& syn = p->h_desc[0][f];
    auto& ana = p->h_desc[1][f];
    syn.clear();
    ana.clear();
    for (int idx : probs) {
      int m = idx / 2, q = idx % 2, s = q ^ f;
      ShtGemmDesc a{};
      a.t_off = p->syn_off[idx];
      a.ldt = p->Hx;
      a.X = p->H;
      a.K = p->e[idx];
      a.d_row = p->cf_row[idx];
      a.c_row = (int64_t)(m * 2 + s) * p->H;
      a.m = m;
      syn.push_back(a);
      ShtGemmDesc b{};
      b.t_off = p->ana_off[idx];
      b.ldt = p->ex[idx];
      b.X = p->e[idx];
      b.K = p->H;
      b.d_row = (int64_t)(m * 2 + s) * p->H;
      b.c_row = p->cf_row[idx];
      b.m = m;
      ana.push_back(b);
    }
  }
  // Item lists: (problem, x-tile) pairs sorted by descending cost, for the
  // plan's tile width and, on FP32 plans, for the narrow variant's.
  auto item_list = [&](int dir, int width, ShtGemmItem** dst, int* count) {
    std::vector<std::pair<int64_t, ShtGemmItem>> items;
    const auto& descs = p->h_desc[dir][0];
    for (int i = 0; i < (int)descs.size(); ++i) {
      const auto& d = descs[i];
      for (int x0 = 0; x0 < d.X; x0 += width) {
        int64_t cost = (int64_t)d.K * std::min(width, d.X - x0);
        items.push_back({cost, ShtGemmItem{i, x0}});
      }
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<ShtGemmItem> flat;
    for (auto& it : items) flat.push_back(it.second);
    *count = (int)flat.size();
    SHT_CUDA_OR_THROW(cudaMalloc(dst, sizeof(ShtGemmItem) * std::max<size_t>(flat.size(), 1)));
    upload_now(*dst, flat.data(), sizeof(ShtGemmItem) * flat.size());
  };
  for (int dir = 0; dir < 2; ++dir) {
    item_list(dir, bx, &p->d_items[dir], &p->n_items[dir]);
    if (p->prec != SHT_PREC_F64)
      item_list(dir, SimtCfg<float, true>::BX, &p->d_items_narrow[dir], &p->n_items_narrow[dir]);
    for (int f = 0; f < 2; ++f) {
      auto& v = p->h_desc[dir][f];
      SHT_CUDA_OR_THROW(cudaMalloc(&p->d_desc[dir][f], sizeof(ShtGemmDesc) * std::max<size_t>(v.size(), 1)));
      upload_now(p->d_desc[dir][f], v.data(), sizeof(ShtGemmDesc) * v.size());
    }
  }
}

template <typename T>
void launch_gemm_simt(const sht_plan* p, int direction, int flip, const T* table, const T* data,
                      T* out, int64_t R, cudaStream_t s) {
  if (p->n_items[direction] == 0 || R == 0) return;
  if constexpr (std::is_same<T, float>::value) {
    if (p->tune_simt_tile == 1) {
      SHT_REQUIRE(p->d_items_narrow[direction] != nullptr, "narrow SIMT work list not built");
      using C = SimtCfg<float, true>;
      dim3 grid((unsigned)p->n_items_narrow[direction], (unsigned)div_up(R, C::BR));
      SHT_REQUIRE(grid.y <= 65535, "too many planes for one launch");
      gemm_simt_kernel<float, true><<<grid, 256, 0, s>>>(
          p->d_desc[direction][flip], p->d_items_narrow[direction], table, data, out, R);
      SHT_CUDA_OR_THROW(cudaGetLastError());
      return;
    }
  }
  using C = SimtCfg<T, false>;
  SHT_REQUIRE(p->gemm_bx == C::BX, "SIMT work list built for another tile width");
  dim3 grid((unsigned)p->n_items[direction], (unsigned)div_up(R, C::BR));
  SHT_REQUIRE(grid.y <= 65535, "too many planes for one launch");
  gemm_simt_kernel<T, false><<<grid, 256, 0, s>>>(p->d_desc[direction][flip], p->d_items[direction],
                                                  table, data, out, R);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

template void launch_gemm_simt<float>(const sht_plan*, int, int, const float*, const float*,
                                      float*, int64_t, cudaStream_t);
template void launch_gemm_simt<double>(const sht_plan*, int, int, const double*, const double*,
                                       double*, int64_t, cudaStream_t);

}  // namespace sht
