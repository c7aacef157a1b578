// Split-precision Legendre contraction on the 5th-generation tensor cores
// (tcgen05, sm_100a).
//
// For every (order m, parity q) block: out[x][r] = sum_k Tab[k][x] D[k][r].
// The MMA sees it as C (M x N) = A (M x K) B^T with
//   M = 128 data rows r (plane x re/im), N = a tile of the table's x extent
//   (<= 256, multiple of 16), K = the contraction (latitude pairs for the
//   analysis, degrees for the synthesis).
// Both operands are split into FP16 hi + lo halves after a power-of-two
// scaling that puts each operand row/column maximum in [2^14, 2^15):
//   A ~ (hi_a + lo_a) / s_r,  B ~ (hi_b + lo_b) / s_x,
//   C = (hi_a hi_b + hi_a lo_b + lo_a hi_b) / (s_r s_x)      (lo*lo dropped)
// accumulated in FP32 in tensor memory.  The table halves and their column
// scales are built once per plan from the FP64 tables and stored in global
// memory as the exact shared-memory image of each (tile, K-stage), so one
// bulk copy per half moves a stage.  The data rows are split on the fly by
// converter warps: a first pass over the tile's K extent finds each row's
// maximum (the per-row, per-order scale), a second converts and stores the
// halves into shared memory.
//
// Roles (448 threads, one CTA per SM, persistent over a cost-sorted tile list):
//   warp 0      bulk-copy loader for the table stages; owns TMEM alloc/free
//   warp 1      MMA issuer (one thread)
//   warps 2-5   epilogue: tcgen05.ld of the accumulator, unscale, store
//   warps 6-13  converters for the data operand
// Pipelines: STAGES shared-memory stages (full/empty mbarriers), two TMEM
// accumulators of 256 columns (full/empty mbarriers), four row-scale slots.
// Every mbarrier wait is bounded by a clock budget; on expiry the thread
// raises the plan's error word, sets a CTA abort flag and every role drains
// and exits, so a fault in the pipeline logic cannot hang the GPU.
//
// Operand layouts are the canonical no-swizzle MN-major UMMA layouts: a core
// matrix is 8 K-rows of 8 contiguous M (or N) elements (16 bytes each row,
// 128 bytes per core matrix); M/N groups are SBO = 128 bytes apart and K
// groups LBO bytes apart.
#include <algorithm>
#include <cmath>

#include "sht_plan.h"

struct ShtTcTile {
  int problem;  // index into the direction's descriptor list
  int n0;       // first x of the tile
  int nsize;    // tile N (multiple of 16, <= 256); 0 for an empty problem
  int kst;      // K stages of BK (0 for an empty problem: the tile writes zeros)
  int r0;       // first data row
  int img;      // index of the tile's (problem, n-tile) image block
};

struct ShtTc16 {
  // Per table kind (basis, dbasis, analysis, rot, shear): the hi/lo images
  // and the per-x column scales (1/s_x), plus per (problem, n-tile) offsets.
  void* img[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float* colscale[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // Per direction: image offsets (bytes) of each (problem, n-tile) block and
  // column-scale offsets (floats) of each problem.
  int64_t* d_img_off[2] = {nullptr, nullptr};
  int64_t* d_cs_off[2] = {nullptr, nullptr};
  std::vector<int64_t> img_off[2], cs_off[2];
  std::vector<int> nt_of[2], nsize_of[2], kst_of[2], img_base[2];
  int64_t img_bytes[2] = {0, 0};
  int64_t cs_elems[2] = {0, 0};
  // Tile lists are built per row count R (cached).
  int64_t tiles_R[2] = {-1, -1};
  ShtTcTile* d_tiles[2] = {nullptr, nullptr};
  int n_tiles[2] = {0, 0};
  int sm_count = 148;
};

namespace sht {
namespace {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int STAGES = 2;
constexpr int NMAX = 256;
constexpr int kThreads = 448;
constexpr int kConvThreads = 256;
constexpr int kConvWarp0 = 6;
constexpr int kEpiWarp0 = 2;
constexpr long long kWaitBudget = 4000000000LL;  // clock cycles (~2 s)

// Shared-memory plan (bytes).
constexpr int kAStage = BM * BK * 2;     // one half of the A stage: 16 KB
constexpr int kBStage = NMAX * BK * 2;   // one half of the B stage: 32 KB
constexpr int kOffA = 0;                                  // [STAGES][2][kAStage]
constexpr int kOffB = kOffA + STAGES * 2 * kAStage;       // [STAGES][2][kBStage]
constexpr int kOffRS = kOffB + STAGES * 2 * kBStage;      // float rowscale[4][128]
constexpr int kOffRed = kOffRS + 4 * BM * 4;              // float red[8][128]
constexpr int kOffBar = kOffRed + 8 * BM * 4;             // mbarriers (8 B each)
constexpr int kNumBars = 3 * STAGES + 4 + 4 + 4 + 1;
constexpr int kOffMisc = kOffBar + kNumBars * 8;          // tmem base, abort flag
constexpr int kSmemBytes = kOffMisc + 16 + 1024;          // + alignment slack

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// No-swizzle shared-memory matrix descriptor (sm_100 version bits = 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: D = F32, A = B = F16, both MN-major.
__device__ __forceinline__ uint32_t instr_desc(int n) {
  return (1u << 4) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

// Power-of-two scale putting a maximum into [2^14, 2^15).
__device__ __forceinline__ float pow2_scale(float mx) {
  if (!(mx > 0.f) || !isfinite(mx)) return 1.f;
  int e;
  frexpf(mx, &e);  // mx = f 2^e, f in [0.5, 1)
  // Clamped so that s and 1/s are normal floats (rows of subnormal values
  // stay tiny, which is all their contribution can be).
  return ldexpf(1.f, max(-126, min(126, 15 - e)));
}

struct TcArgs {
  const ShtGemmDesc* descs;
  const ShtTcTile* tiles;
  int n_tiles;
  const unsigned char* img;
  const int64_t* img_off;  // per (problem, n-tile) block: byte offset of k-stage 0
  const float* colscale;
  const int64_t* cs_off;   // per problem
  const float* data;
  float* out;
  int64_t R;
  unsigned* err;
};

struct Pipe {
  uint64_t* full_a;
  uint64_t* full_b;
  uint64_t* empty;
  uint64_t* acc_full;
  uint64_t* acc_empty;
  uint64_t* rs_free;  // [4]
  uint64_t* rs_full;  // [4]
  uint64_t* done;
  volatile int* abort;
};

// Named-barrier reduction: every thread of the group gets the OR of `v`
// (bar.red also orders shared memory like bar.sync).
__device__ __forceinline__ bool group_any(bool v, int id, int count) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred pi, po;\n\tsetp.ne.u32 pi, %1, 0;\n\t"
      "bar.red.or.pred po, %2, %3, pi;\n\tselp.u32 %0, 1, 0, po;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)v), "r"(id), "r"(count)
      : "memory");
  return out != 0;
}

// Bounded wait: returns false (and raises the abort flag) when the clock
// budget runs out or another role has aborted.
__device__ bool wait_bar(uint64_t* bar, uint32_t parity, const Pipe& pp, unsigned* err, int where) {
  long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*pp.abort) return false;
    if (clock64() - t0 > kWaitBudget) {
      *pp.abort = 1;
      atomicOr(err, kErrMbarTimeout);
      atomicExch(err + 2, (unsigned)where);
      return false;
    }
  }
  return true;
}

__global__ void __launch_bounds__(kThreads, 1) tc_gemm_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte align the working area.
  unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  unsigned char* sA = smem + kOffA;
  unsigned char* sB = smem + kOffB;
  float* rowscale = reinterpret_cast<float*>(smem + kOffRS);
  float* red = reinterpret_cast<float*>(smem + kOffRed);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  uint32_t* tmem_base_smem = reinterpret_cast<uint32_t*>(smem + kOffMisc);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + kOffMisc + 4);
  Pipe pp{bars, bars + STAGES, bars + 2 * STAGES, bars + 3 * STAGES, bars + 3 * STAGES + 2,
          bars + 3 * STAGES + 4, bars + 3 * STAGES + 8, bars + 3 * STAGES + 12, abort_flag};

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&pp.full_a[s], kConvThreads);
      mbar_init(&pp.full_b[s], 1);
      mbar_init(&pp.empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&pp.acc_full[b], 1);
      mbar_init(&pp.acc_empty[b], 128);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&pp.rs_free[b], 128);
      mbar_init(&pp.rs_full[b], 128);
    }
    mbar_init(pp.done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_base_smem, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_base_smem;
  const int64_t R = a.R;

  if (warp == 0) {
    // ------------------------------------------------------------ loader
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int armed[STAGES];
#pragma unroll
      for (int s = 0; s < STAGES; ++s) armed[s] = -1;
      for (int t = blockIdx.x; t < a.n_tiles && !*abort_flag; t += gridDim.x) {
        const ShtTcTile tl = a.tiles[t];
        const int half = tl.nsize * BK * 2;
        const unsigned char* src = a.img + a.img_off[tl.img];
        bool ok = true;
        for (int ks = 0; ks < tl.kst; ++ks) {
          if (!wait_bar(&pp.empty[stage], phase ^ 1, pp, a.err, 1)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&pp.full_b[stage], 2 * half);
          unsigned char* dst = sB + stage * 2 * kBStage;
          bulk_g2s(dst, src + (int64_t)ks * 2 * half, half, &pp.full_b[stage]);
          bulk_g2s(dst + kBStage, src + (int64_t)ks * 2 * half + half, half, &pp.full_b[stage]);
          armed[stage] = (int)phase;
          if (++stage == STAGES) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
      }
      // Drain: the copies of every armed stage land before the CTA exits (in
      // normal operation the MMA has already waited on them; after an abort
      // this wait is what keeps a late copy from writing freed shared memory).
      for (int s = 0; s < STAGES; ++s) {
        if (armed[s] < 0) continue;
        long long t0 = clock64();
        while (!mbar_try_wait(&pp.full_b[s], (uint32_t)armed[s]) && clock64() - t0 < kWaitBudget) {
        }
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool issued = false;
      for (int t = blockIdx.x; t < a.n_tiles && !*abort_flag; t += gridDim.x) {
        const ShtTcTile tl = a.tiles[t];
        if (tl.kst == 0) continue;
        if (!wait_bar(&pp.acc_empty[acc], acc_phase ^ 1, pp, a.err, 2)) break;
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * NMAX);
        const uint32_t idesc = instr_desc(tl.nsize);
        const uint32_t lbo_b = (uint32_t)tl.nsize * 16;
        bool ok = true;
        for (int ks = 0; ks < tl.kst; ++ks) {
          if (!wait_bar(&pp.full_a[stage], phase, pp, a.err, 3) ||
              !wait_bar(&pp.full_b[stage], phase, pp, a.err, 4)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_hi = smem_u32(sA + stage * 2 * kAStage);
          const uint32_t a_lo = a_hi + kAStage;
          const uint32_t b_hi = smem_u32(sB + stage * 2 * kBStage);
          const uint32_t b_lo = b_hi + kBStage;
#pragma unroll
          for (int j = 0; j < BK / 16; ++j) {
            // one K step of 16 = two K groups of 8
            const uint64_t dah = smem_desc(a_hi + j * 2 * 2048, 2048, 128);
            const uint64_t dal = smem_desc(a_lo + j * 2 * 2048, 2048, 128);
            const uint64_t dbh = smem_desc(b_hi + j * 2 * lbo_b, lbo_b, 128);
            const uint64_t dbl = smem_desc(b_lo + j * 2 * lbo_b, lbo_b, 128);
            const uint32_t accum = (ks > 0 || j > 0) ? 1u : 0u;
            mma_f16(d_tmem, dah, dbh, idesc, accum);
            mma_f16(d_tmem, dah, dbl, idesc, 1u);
            mma_f16(d_tmem, dal, dbh, idesc, 1u);
          }
          issued = true;
          mma_commit(&pp.empty[stage]);  // frees the stage when these MMAs finish
          if (++stage == STAGES) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
        mma_commit(&pp.acc_full[acc]);
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
      if (issued) {
        // All issued MMAs complete before TMEM is released.
        mma_commit(pp.done);
        long long t0 = clock64();
        while (!mbar_try_wait(pp.done, 0) && clock64() - t0 < kWaitBudget) {
        }
      }
    }
  } else if (warp < kConvWarp0) {
    // ----------------------------------------------------------- epilogue
    const int eg = warp & 3;  // TMEM lane group accessible to this warp
    const int row = eg * 32 + lane;
    const int et = threadIdx.x - kEpiWarp0 * 32;  // 0..127
    int acc = 0;
    uint32_t acc_phase = 0;
    int ti = 0;  // non-empty tiles seen (row-scale slot = ti & 3)
    // Decisions that gate tcgen05.ld.sync.aligned and the named barriers are
    // made by one elected thread and shared with group_any, so the 128
    // epilogue threads always take the same path.
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
      const ShtTcTile tl = a.tiles[t];
      const ShtGemmDesc d = a.descs[tl.problem];
      const int64_t r = tl.r0 + row;
      float* outb = a.out + d.c_row * R;
      if (tl.kst == 0) {
        // empty contraction (K = 0): the output block is zero
        if (r < R)
          for (int x = tl.n0; x < min(tl.n0 + tl.nsize, d.X); ++x) outb[(int64_t)x * R + r] = 0.f;
        continue;
      }
      bool failed = false;
      if (et == 0)
        failed = !wait_bar(&pp.acc_full[acc], acc_phase, pp, a.err, 5) ||
                 !wait_bar(&pp.rs_full[ti & 3], (ti >> 2) & 1, pp, a.err, 8);
      if (group_any(failed, 2, 128)) break;
      tc_fence_after();
      const float rs = rowscale[(ti & 3) * BM + row];
      mbar_arrive(&pp.rs_free[ti & 3]);
      const float* cs = a.colscale + a.cs_off[tl.problem];
      const uint32_t taddr = tmem_base + ((uint32_t)(eg * 32) << 16) + (uint32_t)(acc * NMAX);
      for (int c0 = 0; c0 < tl.nsize; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + (uint32_t)c0, v);
        if (r < R) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int x = tl.n0 + c0 + i;
            if (x < d.X) outb[(int64_t)x * R + r] = v[i] * rs * cs[x];
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&pp.acc_empty[acc]);
      if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      ++ti;
    }
  } else {
    // --------------------------------------------------------- converters
    const int ct = threadIdx.x - kConvWarp0 * 32;  // 0..255
    int stage = 0;
    uint32_t phase = 0;
    int ti = 0;  // non-empty tiles seen (row-scale slot = ti & 3)
    for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
      const ShtTcTile tl = a.tiles[t];
      if (tl.kst == 0) continue;
      const ShtGemmDesc d = a.descs[tl.problem];
      const float* Db = a.data + d.d_row * R;
      // Row-scale slot ti & 3 must be free (its epilogue has read it).  One
      // elected thread waits; the group-wide reduction is also the barrier
      // that keeps this tile's writes of red[] behind every converter's read
      // of the previous tile's scales.
      bool failed = false;
      if (ct == 0) failed = !wait_bar(&pp.rs_free[ti & 3], ((ti >> 2) & 1) ^ 1, pp, a.err, 6);
      if (group_any(failed, 1, kConvThreads)) break;
      {
        const int rq = (ct & 31) * 4;
        const int kg = ct >> 5;
        float mx[4] = {0.f, 0.f, 0.f, 0.f};
        const int64_t rr = tl.r0 + rq;
        for (int k = kg; k < d.K; k += 8) {
          const float* p = Db + (int64_t)k * R + rr;
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if (rr + i < R) mx[i] = fmaxf(mx[i], fabsf(__ldg(p + i)));
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) red[kg * BM + rq + i] = mx[i];
        asm volatile("bar.sync 1, %0;" ::"n"(kConvThreads));
        if (ct < BM) {
          float m = 0.f;
#pragma unroll
          for (int g = 0; g < 8; ++g) m = fmaxf(m, red[g * BM + ct]);
          const float s = pow2_scale(m);
          rowscale[(ti & 3) * BM + ct] = 1.f / s;  // the epilogue multiplies by 1/s_r
          red[ct] = s;                             // the converters multiply by s_r
          mbar_arrive(&pp.rs_full[ti & 3]);        // publishes the slot to the epilogue
        }
        asm volatile("bar.sync 1, %0;" ::"n"(kConvThreads));
      }
      // Pass 2: convert K stages. Thread: (kk = ct % 8, 8-row group mg = (ct/8) % 16),
      // K groups kg = ct/128 + 2j.
      const int kk = ct & 7, mg = (ct >> 3) & 15, kgs = ct >> 7;
      float sc[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) sc[i] = red[mg * 8 + i];
      const int64_t rbase = tl.r0 + mg * 8;
      const bool full_rows = rbase + 8 <= R && (R % 4) == 0;
      bool ok = true;
      for (int ks = 0; ks < tl.kst; ++ks) {
        bool f = false;
        if (ct == 0) f = !wait_bar(&pp.empty[stage], phase ^ 1, pp, a.err, 7);
        if (group_any(f, 1, kConvThreads)) {
          ok = false;
          break;
        }
        unsigned char* dhi = sA + stage * 2 * kAStage;
        unsigned char* dlo = dhi + kAStage;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int kg = kgs + 2 * j;
          const int k = ks * BK + kg * 8 + kk;
          float v[8];
          if (k < d.K) {
            const float* p = Db + (int64_t)k * R + rbase;
            if (full_rows) {
              const float4 u0 = __ldg(reinterpret_cast<const float4*>(p));
              const float4 u1 = __ldg(reinterpret_cast<const float4*>(p + 4));
              v[0] = u0.x; v[1] = u0.y; v[2] = u0.z; v[3] = u0.w;
              v[4] = u1.x; v[5] = u1.y; v[6] = u1.z; v[7] = u1.w;
            } else {
#pragma unroll
              for (int i = 0; i < 8; ++i) v[i] = (rbase + i < R) ? __ldg(p + i) : 0.f;
            }
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = 0.f;
          }
          __align__(16) __half hi[8];
          __align__(16) __half lo[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float x = v[i] * sc[i];
            hi[i] = __float2half_rn(x);
            lo[i] = __float2half_rn(x - __half2float(hi[i]));
          }
          const int off = kg * 2048 + mg * 128 + kk * 16;
          *reinterpret_cast<uint4*>(dhi + off) = *reinterpret_cast<const uint4*>(hi);
          *reinterpret_cast<uint4*>(dlo + off) = *reinterpret_cast<const uint4*>(lo);
        }
        fence_proxy_async();
        mbar_arrive(&pp.full_a[stage]);
        if (++stage == STAGES) { stage = 0; phase ^= 1; }
      }
      if (!ok) break;
      ++ti;
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem_base, 512);
}

// ------------------------------------------------------- table images
// One thread per (problem, x): the column scale s_x from the maximum of the
// FP64 table over the K extent.
struct ImgArgs {
  const ShtGemmDesc* descs;  // FP64-layout descriptors (t_off, ldt, X, K)
  int n_problems;
  const double* tab;         // FP64 table, [k][x] with ld = ldt
  const int64_t* cs_off;
  float* colscale;           // 1/s_x
  float* colmul;             // s_x (scratch)
};

__global__ void colscale_kernel(ImgArgs a) {
  const int p = blockIdx.y;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_problems) return;
  const ShtGemmDesc d = a.descs[p];
  if (x >= d.X) return;
  double mx = 0.0;
  const double* t = a.tab + d.t_off;
  for (int k = 0; k < d.K; ++k) mx = fmax(mx, fabs(t[(int64_t)k * d.ldt + x]));
  float s = 1.f;
  if (mx > 0.0) {
    int e;
    frexp(mx, &e);
    // Polar values of high orders underflow toward 1e-300: clamp so that s
    // and 1/s stay normal floats; such columns contribute nothing anyway.
    s = ldexpf(1.f, max(-126, min(126, 15 - e)));
  }
  a.colscale[a.cs_off[p] + x] = 1.f / s;
  a.colmul[a.cs_off[p] + x] = s;
}

struct BlockInfo {
  int problem, n0, nsize, kst;
  int64_t off;  // byte offset of the block's image
};

// One thread per image element of one (problem, n-tile) block; the image is
// [k-stage][hi|lo][kg 8][ng nsize/8][kk 8][nn 8] halves.
__global__ void image_kernel(ImgArgs a, const BlockInfo* blocks, int nblocks, unsigned char* img) {
  const int b = blockIdx.y;
  if (b >= nblocks) return;
  const BlockInfo bi = blocks[b];
  const ShtGemmDesc d = a.descs[bi.problem];
  const int64_t per_stage = (int64_t)bi.nsize * BK;  // halves per half-image
  const int64_t total = per_stage * bi.kst;
  __half* base = reinterpret_cast<__half*>(img + bi.off);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int ks = (int)(e / per_stage);
    int rem = (int)(e % per_stage);
    const int nn = rem & 7;
    rem >>= 3;
    const int kk = rem & 7;
    rem >>= 3;
    const int ng = rem % (bi.nsize / 8);
    const int kg = rem / (bi.nsize / 8);
    const int x = bi.n0 + ng * 8 + nn;
    const int k = ks * BK + kg * 8 + kk;
    float hi = 0.f, lo = 0.f;
    if (x < d.X && k < d.K) {
      const double v = a.tab[d.t_off + (int64_t)k * d.ldt + x] * (double)a.colmul[a.cs_off[bi.problem] + x];
      const __half h = __float2half_rn((float)v);
      hi = __half2float(h);
      lo = (float)(v - (double)hi);
    }
    const int64_t pos = ((int64_t)(kg * (bi.nsize / 8) + ng) * 8 + kk) * 8 + nn;
    base[(int64_t)ks * 2 * per_stage + pos] = __float2half_rn(hi);
    base[(int64_t)ks * 2 * per_stage + per_stage + pos] = __float2half_rn(lo);
  }
}

void tile_shape(int X, int& nt, int& nsize) {
  int xp = (int)round_up(std::max(X, 1), 16);
  nt = (int)div_up(xp, NMAX);
  nsize = (int)round_up(div_up(xp, nt), 16);
}

}  // namespace

void build_tc_tables(sht_plan* p, const double* basis64, const double* dbasis64,
                     const double* analysis64, const double* rot64, const double* shear64,
                     cudaStream_t s) {
  ShtTc16* tc = new ShtTc16();
  try {
    int dev = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&dev));
    SHT_CUDA_OR_THROW(cudaDeviceGetAttribute(&tc->sm_count, cudaDevAttrMultiProcessorCount, dev));
    // FP64-layout descriptors of both directions (same construction as the
    // SIMT work list, flip 0; the image depends only on the table block).
    const int T = p->T;
    std::vector<ShtGemmDesc> d64[2];
    for (int m = 0; m <= T; ++m)
      for (int q = 0; q < 2; ++q) {
        int idx = m * 2 + q;
        ShtGemmDesc sy{};
        sy.t_off = p->syn_off[idx];
        sy.ldt = p->Hx;
        sy.X = p->H;
        sy.K = p->e[idx];
        d64[0].push_back(sy);
        ShtGemmDesc an{};
        an.t_off = p->ana_off[idx];
        an.ldt = p->ex[idx];
        an.X = p->e[idx];
        an.K = p->H;
        d64[1].push_back(an);
      }
    const double* tabs[5] = {basis64, dbasis64, analysis64, rot64, shear64};
    const int tab_dir[5] = {0, 0, 1, 1, 1};
    std::vector<BlockInfo> blocks[2];
    for (int dir = 0; dir < 2; ++dir) {
      const int np = (int)d64[dir].size();
      tc->nt_of[dir].resize(np);
      tc->nsize_of[dir].resize(np);
      tc->kst_of[dir].resize(np);
      tc->img_base[dir].resize(np);
      tc->cs_off[dir].resize(np);
      int64_t off = 0, cso = 0;
      for (int i = 0; i < np; ++i) {
        const auto& d = d64[dir][i];
        int nt, ns;
        tile_shape(d.X, nt, ns);
        const int kst = (int)div_up(d.K, BK);
        tc->nt_of[dir][i] = nt;
        tc->nsize_of[dir][i] = ns;
        tc->kst_of[dir][i] = kst;
        tc->img_base[dir][i] = (int)tc->img_off[dir].size();
        tc->cs_off[dir][i] = cso;
        cso += round_up(std::max(d.X, 1), 16);
        for (int j = 0; j < nt; ++j) {
          tc->img_off[dir].push_back(off);
          if (d.X > 0 && kst > 0) blocks[dir].push_back({i, j * ns, ns, kst, off});
          off += (int64_t)kst * 2 * ns * BK * 2;
        }
      }
      tc->img_bytes[dir] = off;
      tc->cs_elems[dir] = cso;
      SHT_CUDA_OR_THROW(cudaMalloc(&tc->d_img_off[dir], 8 * std::max<size_t>(tc->img_off[dir].size(), 1)));
      SHT_CUDA_OR_THROW(cudaMemcpy(tc->d_img_off[dir], tc->img_off[dir].data(),
                                   8 * tc->img_off[dir].size(), cudaMemcpyHostToDevice));
      SHT_CUDA_OR_THROW(cudaMalloc(&tc->d_cs_off[dir], 8 * np));
      SHT_CUDA_OR_THROW(cudaMemcpy(tc->d_cs_off[dir], tc->cs_off[dir].data(), 8 * np,
                                   cudaMemcpyHostToDevice));
    }
    ShtGemmDesc* dd[2];
    BlockInfo* db[2];
    float* colmul[2];
    for (int dir = 0; dir < 2; ++dir) {
      SHT_CUDA_OR_THROW(cudaMalloc(&dd[dir], sizeof(ShtGemmDesc) * d64[dir].size()));
      SHT_CUDA_OR_THROW(cudaMemcpy(dd[dir], d64[dir].data(), sizeof(ShtGemmDesc) * d64[dir].size(),
                                   cudaMemcpyHostToDevice));
      SHT_CUDA_OR_THROW(cudaMalloc(&db[dir], sizeof(BlockInfo) * std::max<size_t>(blocks[dir].size(), 1)));
      SHT_CUDA_OR_THROW(cudaMemcpy(db[dir], blocks[dir].data(), sizeof(BlockInfo) * blocks[dir].size(),
                                   cudaMemcpyHostToDevice));
      SHT_CUDA_OR_THROW(cudaMalloc(&colmul[dir], 4 * std::max<int64_t>(tc->cs_elems[dir], 1)));
    }
    for (int kind = 0; kind < 5; ++kind) {
      const int dir = tab_dir[kind];
      SHT_CUDA_OR_THROW(cudaMalloc(&tc->img[kind], std::max<int64_t>(tc->img_bytes[dir], 16)));
      SHT_CUDA_OR_THROW(cudaMalloc(&tc->colscale[kind], 4 * std::max<int64_t>(tc->cs_elems[dir], 1)));
      ImgArgs ia{dd[dir], (int)d64[dir].size(), tabs[kind], tc->d_cs_off[dir], tc->colscale[kind],
                 colmul[dir]};
      int xmax = 0;
      for (auto& d : d64[dir]) xmax = std::max(xmax, d.X);
      colscale_kernel<<<dim3((unsigned)div_up(std::max(xmax, 1), 128), (unsigned)d64[dir].size()), 128, 0, s>>>(ia);
      if (!blocks[dir].empty())
        image_kernel<<<dim3(64, (unsigned)blocks[dir].size()), 256, 0, s>>>(
            ia, db[dir], (int)blocks[dir].size(), (unsigned char*)tc->img[kind]);
      SHT_CUDA_OR_THROW(cudaGetLastError());
      SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
    }
    for (int dir = 0; dir < 2; ++dir) {
      cudaFree(dd[dir]);
      cudaFree(db[dir]);
      cudaFree(colmul[dir]);
    }
    SHT_CUDA_OR_THROW(cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemBytes));
  } catch (...) {
    p->tc = tc;
    destroy_tc_tables(p);
    throw;
  }
  p->tc = tc;
}

void destroy_tc_tables(sht_plan* p) {
  ShtTc16* tc = p->tc;
  if (!tc) return;
  for (int k = 0; k < 5; ++k) {
    if (tc->img[k]) cudaFree(tc->img[k]);
    if (tc->colscale[k]) cudaFree(tc->colscale[k]);
  }
  for (int d = 0; d < 2; ++d) {
    if (tc->d_img_off[d]) cudaFree(tc->d_img_off[d]);
    if (tc->d_cs_off[d]) cudaFree(tc->d_cs_off[d]);
    if (tc->d_tiles[d]) cudaFree(tc->d_tiles[d]);
  }
  delete tc;
  p->tc = nullptr;
}

void launch_gemm_tc(const sht_plan* p, int direction, int flip, int table_kind, const float* data,
                    float* out, int64_t R, cudaStream_t s) {
  ShtTc16* tc = p->tc;
  SHT_REQUIRE(tc != nullptr, "tensor-core tables not built");
  if (R == 0) return;
  const int dir = direction;
  if (tc->tiles_R[dir] != R) {
    // Tiles: every (problem, n-tile) x every 128-row block, cost-sorted.
    std::vector<std::pair<int64_t, ShtTcTile>> v;
    const int np = (int)tc->nt_of[dir].size();
    for (int i = 0; i < np; ++i) {
      const int nt = tc->nt_of[dir][i], ns = tc->nsize_of[dir][i], kst = tc->kst_of[dir][i];
      const int X = p->h_desc[dir][0][i].X;
      if (X == 0) continue;
      for (int j = 0; j < nt; ++j)
        for (int64_t r0 = 0; r0 < R; r0 += BM) {
          ShtTcTile t{i, j * ns, ns, kst, (int)r0, tc->img_base[dir][i] + j};
          int64_t cost = (int64_t)ns * kst * BK + 4096;
          v.push_back({cost, t});
        }
    }
    std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<ShtTcTile> flat;
    for (auto& e : v) flat.push_back(e.second);
    if (tc->d_tiles[dir]) cudaFree(tc->d_tiles[dir]);
    SHT_CUDA_OR_THROW(cudaMalloc(&tc->d_tiles[dir], sizeof(ShtTcTile) * std::max<size_t>(flat.size(), 1)));
    SHT_CUDA_OR_THROW(cudaMemcpy(tc->d_tiles[dir], flat.data(), sizeof(ShtTcTile) * flat.size(),
                                 cudaMemcpyHostToDevice));
    tc->n_tiles[dir] = (int)flat.size();
    tc->tiles_R[dir] = R;
  }
  if (tc->n_tiles[dir] == 0) return;
  TcArgs a{};
  a.descs = p->d_desc[dir][flip];
  a.tiles = tc->d_tiles[dir];
  a.n_tiles = tc->n_tiles[dir];
  a.img = (const unsigned char*)tc->img[table_kind];
  a.img_off = tc->d_img_off[dir];
  a.colscale = tc->colscale[table_kind];
  a.cs_off = tc->d_cs_off[dir];
  a.data = data;
  a.out = out;
  a.R = R;
  a.err = p->d_err;
  const int grid = std::min(tc->n_tiles[dir], tc->sm_count);
  tc_gemm_kernel<<<grid, kThreads, kSmemBytes, s>>>(a);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

}  // namespace sht
