// Split-precision Legendre contraction on the 5th-generation tensor cores
// (tcgen05, sm_100a).
//
// For every (order m, parity q) block: out[x][r] = sum_k Tab[k][x] D[k][r].
// The MMA sees it as C (M x N) = A (M x K) B^T with
//   M = 128 data rows r (plane x re/im), N = a tile of the table's x extent
//   (<= 128, multiple of 16), K = the contraction (latitude pairs for the
//   analysis, degrees for the synthesis).
// Both operands are split into two FP16 parts after a power-of-two scaling
// that puts each data row / table column maximum in [2^14, 2^15):
//   a s_r = a1 + a2,  b s_x = b1 + b2            (11 significant bits each)
//   C = (a1 b1 + [a1 b2 + a2 b1]) / (s_r s_x)
// The main product a1 b1 accumulates in NMAIN = 3 TMEM accumulators, one per
// contiguous third of the K steps, and the two correction products in a
// fourth; the epilogue adds the four in FP32.  The tensor core's FP32
// accumulate truncates: with all three products in one accumulator every
// correction step adds another truncation of the full-size sum (1.3e-6
// relative spectral L2 at T255, in an emulation of the pipeline), with the
// correction separated the main sum's own truncations remain (1.2e-6 at
// T511 measured), and splitting the main sum into three segments cuts their
// growth (3.6e-7 at T511 measured; the plain FP32 path measures 2.9e-7).  The table parts and the column scales are
// built once per plan from the FP64 tables and stored as the exact
// shared-memory image of each (tile, K-stage), so one bulk copy per part
// moves a stage.  The data rows are split on the fly by converter warps;
// their row scales come from the row maxima the producing kernel (the
// longitude FFT or the pack kernel) merged while writing the operand.
//
// Roles (576 threads, one CTA per SM, persistent over a cost-sorted tile list
// that may merge several contractions: the P and dP/dphi tables of a
// gradient or wind synthesis, or the plans of a batch):
//   warp 0      bulk-copy loader for the table stages; owns TMEM alloc/free
//   warp 1      MMA issuer (one thread)
//   warps 2-9   epilogue: tcgen05.ld of the accumulators, unscale, release
//               the accumulators, store the tile to global memory
//   warps 10-17 converters for the data operand (into shared memory, or into
//               TMEM for the kTmemA plan)
// Pipelines: S shared-memory stages (full/empty mbarriers), NA data-operand
// slots (the shared stages themselves, or TMEM slots with their own
// full/empty mbarriers) and one or two
// sets of TMEM accumulators of 128 columns each (full/empty mbarriers per set).  Every
// mbarrier wait is bounded by a clock budget; on expiry the waiting thread
// raises the plan's error word and a CTA abort flag, and the epilogue warps
// decide to stop together (a reduction over their named barrier) before the
// warp-collective TMEM loads, so a fault in the pipeline logic cannot hang
// the GPU.
//
// Operand layouts are the canonical no-swizzle MN-major UMMA layouts: a core
// matrix is 8 K-rows of 8 contiguous M (or N) elements (16 bytes each row,
// 128 bytes per core matrix); M/N groups are SBO = 128 bytes apart and K
// groups LBO bytes apart.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include <cuda.h>  // CUtensorMap (the tensor map is encoded through the runtime's driver entry point)

#include "sht_plan.h"

// One tile of a launch, self-contained: every role reads one 64-byte record
// per tile (staged in shared memory per CTA) instead of a chain of dependent
// global loads (tile -> descriptor -> image offset) at each tile start.
struct alignas(16) ShtTcTile {
  int group;      // index into the launch's group list
  int problem;    // index into the direction's descriptor list
  int n0;         // first x of the tile
  int nsize;      // tile N (multiple of 16, <= 128); 0 for an empty problem
  int kst;        // K stages of BK (0 for an empty problem: the tile writes zeros)
  int r0;         // first data row
  int X;          // the problem's output extent (columns past it are not stored)
  int K;          // the problem's contraction extent
  int64_t img;    // byte offset of the tile's table image (k-stage 0)
  int64_t d_row;  // data row of the problem's k = 0
  int64_t c_row;  // output row of the problem's x = 0
  int64_t cs;     // column-scale index of the problem's x = 0
};
static_assert(sizeof(ShtTcTile) == 64, "tile records are 64 bytes");

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
  // Tile lists of this plan's own launches.
  sht::TcTileCache* tiles = nullptr;
  int sm_count = 148;
};

namespace sht {
namespace {

constexpr int BM = 128;
constexpr int BK = 32;
constexpr int NPARTS = 2;
constexpr int NMAX = 128;   // tile N
constexpr int kMaxNBuf = 2;
// Roles: warp 0 table loader (and TMEM owner), warp 1 MMA issuer, warps 2-9
// the epilogue (two per TMEM lane quarter), warps 10-17 the converters,
// warp 18 the data-tile TMA loader.
constexpr int kEpiWarp0 = 2;
constexpr int kEpiWarps = 8;
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kConvThreads = 256;
constexpr int kConvWarp0 = kEpiWarp0 + kEpiWarps;
constexpr int kRawWarp = kConvWarp0 + kConvThreads / 32;
constexpr int kThreads = (kRawWarp + 1) * 32;  // 608
constexpr long long kWaitBudget = 4000000000LL;  // clock cycles (~2 s)
// Per-CTA staging in shared memory: the CTA's tile records (when it has at
// most kMaxCtaTiles) and the power-of-two row scales of every group (when the
// launch has at most kMaxRowScales data rows); larger launches read both from
// global memory.
constexpr int kMaxCtaTiles = 192;
constexpr int kMaxRowScales = 2048;

// Shared-memory pieces (bytes).
constexpr int kAPart = BM * BK * 2;      // one FP16 part of the A stage: 8 KB
constexpr int kBPart = NMAX * BK * 2;    // one FP16 part of the B stage: 8 KB
constexpr int kALbo = (BM / 8) * 128;    // A: K-group stride (16 M-groups of 128 B)
constexpr int kRawStage = BK * BM * 4;   // FP32 data tile of a stage: 16 KB
constexpr int kRawBox = BK * 32 * 4;     // one TMA box: 32 rows x 32 k, 4 KB

// TMEM accumulator plans (SHT_TUNE_ACCUMULATORS).  kAccurate: the main
// product in three K-segment accumulators + corrections, one set (512
// columns).  kOverlapped: one main accumulator + corrections, two sets, so the
// epilogue drains one tile while the MMA fills the next (faster; the longer
// truncated main sums raise the split error from about 3.6e-7 to 1.2e-6).
// kTmemA: two K-segment accumulators + corrections (384 columns) and the
// converted data operand in the other 128 TMEM columns, so the MMA reads only
// the table operand from shared memory (split error ~6e-7 at T511).
template <int NMAIN_, int NBUF_, bool A_TMEM_ = false>
struct AccPlan {
  static constexpr int NMAIN = NMAIN_;  // main-product accumulators (contiguous K segments)
  static constexpr int NBUF = NBUF_;    // accumulator sets
  static constexpr int kAccCols = (NMAIN + 1) * NMAX;  // one set: NMAIN mains + corrections
  // A_TMEM: the data operand's hi and lo FP16 parts (16 columns each per
  // slot) live in TMEM after the accumulators.
  static constexpr bool A_TMEM = A_TMEM_;
  // Six shared stages with four TMEM slots measured slower than four and
  // four (the extra slot commit per stage; the table loads are bandwidth-,
  // not depth-limited), so both plans run four.
  static constexpr int S = 4;   // shared stages: table (+ raw data) (+ A)
  static constexpr int NA = 4;  // data-operand slots (TMEM or shared)
  static constexpr int kATmem = NBUF * kAccCols;  // first A column in TMEM
  static_assert(kATmem + (A_TMEM ? NA * 32 : 0) <= 512, "TMEM holds 512 columns");
  // Shared-memory plan.
  static constexpr int kOffA = 0;                                             // [NA][NPARTS][kAPart]
  static constexpr int kOffB = kOffA + (A_TMEM ? 0 : NA * NPARTS * kAPart);   // [S][NPARTS][kBPart]
  static constexpr int kOffRaw = kOffB + S * NPARTS * kBPart;                 // [S][4 boxes], swizzled
  static constexpr int kOffBar = kOffRaw + S * kRawStage;                     // mbarriers (8 B each)
  static constexpr int kNumBars = 4 * S + 2 * NA + 2 * kMaxNBuf + 1;
  static_assert(kOffRaw % 1024 == 0, "128-byte swizzled TMA destinations are 1024-byte aligned");
  static constexpr int kOffMisc = kOffBar + kNumBars * 8;           // tmem base, abort flag
  static constexpr int kOffCs = (kOffMisc + 16 + 127) / 128 * 128;  // [epilogue warps][NMAX] floats
  static constexpr int kOffTiles = kOffCs + kEpiWarps * NMAX * 4;     // [kMaxCtaTiles] tile records
  static constexpr int kOffRs = kOffTiles + kMaxCtaTiles * (int)sizeof(ShtTcTile);  // row scales
  static constexpr int kSmemBytes = kOffRs + kMaxRowScales * 4 + 1024;  // + alignment slack
  static_assert(kSmemBytes <= 227 * 1024, "shared memory plan exceeds 227 KB");
};
using kAccurate = AccPlan<3, 1>;
using kOverlapped = AccPlan<1, 2>;
using kTmemA = AccPlan<2, 1, true>;

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
// TMA: one 2D box of the data operand (x = data row r, y = contraction row k)
// into shared memory, completing on `bar`.  Boxes that reach past the
// tensor's extent are zero-filled by the hardware.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Named barrier 1 over the eight epilogue warps; returns the OR of `pred`
// over their 256 threads.
__device__ __forceinline__ bool epi_bar_or(bool pred) {
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.or.pred p, 1, 256, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(out)
      : "r"((uint32_t)pred)
      : "memory");
  return out != 0;
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
// The same with A from tensor memory (K-major: row m in lane m, two FP16 K
// values per 32-bit column, the even one in the low half).
__device__ __forceinline__ void mma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc,
                                           uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// tcgen05.st of 8 consecutive columns of this warp's 32 lanes, and the wait
// for this thread's stores.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// tcgen05.ld of 16 consecutive columns, without the wait: the registers are
// valid only after tmem_wait16 below.
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// tcgen05.wait::ld (when WAIT) and a register dependency on r, so that no
// use of r can be scheduled before the wait.
template <bool WAIT>
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
  if constexpr (WAIT) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
  } else {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                   "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                   "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
  }
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

// x rounded to 11 significant bits (the FP16 significand), ties away from
// zero, by integer arithmetic on the FP32 encoding: the high FP16 part of
// the split without a float -> half -> float round trip (conversions run at
// a fraction of the FP32 rate and were the converter warps' bottleneck).
// Values scaled into FP16's normal range convert to FP16 exactly; below it
// the FP16 rounding error is under 2^-24 absolute, 2^-38 of the row maximum.
__device__ __forceinline__ float round_to_11_bits(float x) {
  return __int_as_float((__float_as_int(x) + 0x1000) & ~0x1FFF);
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

// One contraction of a launch: a table (one direction of one plan), the data
// operand with its row maxima, and the output.  A launch runs the merged,
// cost-sorted tiles of up to kMaxTcGroups of them.
struct alignas(64) TcGroup {
  CUtensorMap data_map;    // the data operand as a [rows][R] FP32 tensor (when use_tma)
  int use_tma;             // 1: the loader brings the data tiles in by TMA
  const unsigned char* img;
  const float* colscale;
  const float* data;
  const float* rowmax;     // per data row: max |value| (from the producer kernel)
  float* out;
  int64_t R;
  int rs_off;              // first entry of this group's row scales in shared memory
};

struct TcArgs {
  TcGroup g[kMaxTcGroups];
  const ShtTcTile* tiles;
  int n_tiles;
  int stage_rs;            // 1: the launch's row scales fit in shared memory
  int rs_total;            // their count
  unsigned* err;
};

struct Pipe {
  uint64_t* full_a;    // [NA] the data operand of a slot is converted
  uint64_t* full_b;    // [S]
  uint64_t* empty;     // [S] the MMAs of a shared stage are done
  uint64_t* full_raw;  // [S] the FP32 data tile of a raw stage has landed (TMA)
  uint64_t* a_empty;   // [NA] the MMAs of a TMEM data slot are done (A_TMEM)
  uint64_t* acc_full;   // [kMaxNBuf]
  uint64_t* acc_empty;  // [kMaxNBuf]
  uint64_t* done;
  uint64_t* raw_empty;  // [S] the converters have read a raw stage
  volatile int* abort;
};

// A tile whose fields could make a TMA load, an MMA or an address invalid
// (row offset not a multiple of 32, group or width out of range) is never
// issued: the role that reads it raises kErrBadTile and the abort flag.
__device__ __forceinline__ bool tile_ok(const ShtTcTile& tl) {
  return tl.group >= 0 && tl.group < kMaxTcGroups && tl.r0 >= 0 && (tl.r0 & 31) == 0 &&
         tl.kst >= 0 && tl.nsize >= 0 && tl.nsize <= NMAX && (tl.nsize & 15) == 0 &&
         (tl.kst == 0 || tl.nsize >= 16);
}
__device__ __forceinline__ bool reject_tile(const ShtTcTile& tl, volatile int* abort_flag,
                                            unsigned* err) {
  if (tile_ok(tl)) return false;
  *abort_flag = 1;
  atomicOr(err, kErrBadTile);
  return true;
}

__device__ bool wait_bar(uint64_t* bar, uint32_t parity, const Pipe& pp, unsigned* err, int where);
// The common case inline: the phase has already completed.
__device__ __forceinline__ bool wait_fast(uint64_t* bar, uint32_t parity, const Pipe& pp,
                                          unsigned* err, int where) {
  return mbar_try_wait(bar, parity) || wait_bar(bar, parity, pp, err, where);
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

// 576 threads = 18 warps, 5 on the busiest of the four SM sub-partitions,
// whose 16 384 registers cap a thread at 96.
template <typename Acc>
__global__ void __launch_bounds__(kThreads, 1) tc_gemm_kernel(const __grid_constant__ TcArgs a) {
  constexpr int NMAIN = Acc::NMAIN, NBUF = Acc::NBUF, kAccCols = Acc::kAccCols;
  constexpr int S = Acc::S, NA = Acc::NA;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte align the working area.
  unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
  unsigned char* sA = smem + Acc::kOffA;
  unsigned char* sB = smem + Acc::kOffB;
  unsigned char* sRaw = smem + Acc::kOffRaw;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Acc::kOffBar);
  uint32_t* tmem_base_smem = reinterpret_cast<uint32_t*>(smem + Acc::kOffMisc);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(smem + Acc::kOffMisc + 4);
  Pipe pp{bars,
          bars + NA,
          bars + NA + S,
          bars + NA + 2 * S,
          bars + NA + 3 * S,
          bars + 2 * NA + 3 * S,
          bars + 2 * NA + 3 * S + kMaxNBuf,
          bars + 2 * NA + 3 * S + 2 * kMaxNBuf,
          bars + 2 * NA + 3 * S + 2 * kMaxNBuf + 1,
          abort_flag};

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NA; ++s) {
      mbar_init(&pp.full_a[s], kConvThreads);
      mbar_init(&pp.a_empty[s], 1);
    }
    for (int s = 0; s < S; ++s) {
      mbar_init(&pp.full_b[s], 1);
      mbar_init(&pp.empty[s], 1);
      mbar_init(&pp.full_raw[s], 1);
      mbar_init(&pp.raw_empty[s], kConvThreads / 32);
    }
    for (int b = 0; b < kMaxNBuf; ++b) {
      mbar_init(&pp.acc_full[b], 1);
      mbar_init(&pp.acc_empty[b], kEpiThreads);
    }
    mbar_init(pp.done, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(tmem_base_smem, 512);
    tmem_relinquish();
  }
  // This CTA's tile records and the launch's row scales, staged once.
  ShtTcTile* s_tiles = reinterpret_cast<ShtTcTile*>(smem + Acc::kOffTiles);
  float* s_rs = reinterpret_cast<float*>(smem + Acc::kOffRs);
  const int my_tiles = (int)blockIdx.x < a.n_tiles ? (a.n_tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const bool staged = my_tiles <= kMaxCtaTiles;
  if (staged) {
    const uint4* src = reinterpret_cast<const uint4*>(a.tiles);
    uint4* dst = reinterpret_cast<uint4*>(s_tiles);
    for (int e = threadIdx.x; e < my_tiles * 4; e += blockDim.x)
      dst[e] = src[((int64_t)blockIdx.x + (int64_t)(e >> 2) * gridDim.x) * 4 + (e & 3)];
  }
  if (a.stage_rs) {
#pragma unroll 1
    for (int gi = 0; gi < kMaxTcGroups; ++gi) {
      const TcGroup& G = a.g[gi];
      for (int64_t r = threadIdx.x; r < G.R; r += blockDim.x) s_rs[G.rs_off + r] = pow2_scale(G.rowmax[r]);
    }
  }
  // The k-th tile of this CTA (tile index blockIdx.x + k * gridDim.x).
  auto tile_k = [&](int k) -> ShtTcTile {
    return staged ? s_tiles[k] : a.tiles[(int64_t)blockIdx.x + (int64_t)k * gridDim.x];
  };
  // Power-of-two scale of data row r (< R) of a group.
  auto row_scale = [&](const TcGroup& G, int64_t r) -> float {
    return a.stage_rs ? s_rs[G.rs_off + r] : pow2_scale(G.rowmax[r]);
  };
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_base_smem;

  if (warp == 0) {
    // ------------------------------------------------------------ loader
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int armed[S];
#pragma unroll
      for (int s = 0; s < S; ++s) armed[s] = -1;
      for (int k = 0; k < my_tiles && !*abort_flag; ++k) {
        const ShtTcTile tl = tile_k(k);
        if (reject_tile(tl, abort_flag, a.err)) break;
        const TcGroup& G = a.g[tl.group];
        const int part = tl.nsize * BK * 2;  // bytes of one FP16 part of one stage
        const unsigned char* src = G.img + tl.img;
        bool ok = true;
        for (int ks = 0; ks < tl.kst; ++ks) {
          if (!wait_bar(&pp.empty[stage], phase ^ 1, pp, a.err, 1)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&pp.full_b[stage], NPARTS * part);
          unsigned char* dst = sB + stage * NPARTS * kBPart;
#pragma unroll
          for (int pt = 0; pt < NPARTS; ++pt)
            bulk_g2s(dst + pt * kBPart, src + ((int64_t)ks * NPARTS + pt) * part, part,
                     &pp.full_b[stage]);
          armed[stage] = (int)phase;
          if (++stage == S) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
      }
      // Drain: the copies of every armed stage land before the CTA exits (in
      // normal operation the MMA has already waited on them; after an abort
      // this wait is what keeps a late copy from writing freed shared memory).
      for (int s = 0; s < S; ++s) {
        long long t0 = clock64();
        if (armed[s] >= 0)
          while (!mbar_try_wait(&pp.full_b[s], (uint32_t)armed[s]) && clock64() - t0 < kWaitBudget) {
          }
      }
    }
  } else if (warp == kRawWarp) {
    // ---------------------------------------------------- data-tile loader
    // The FP32 data tiles by TMA into their own ring of S raw stages, each
    // refilled as soon as the converters have read it (not when the MMAs of
    // its stage finish): the data runs up to S stages ahead of the converted
    // operand ring, which is what keeps the tensor pipe fed across the
    // memory latency.
    if (lane == 0 && a.g[0].use_tma) {
      int stage = 0;
      uint32_t phase = 0;
      int armed[S];
#pragma unroll
      for (int s = 0; s < S; ++s) armed[s] = -1;
      for (int k = 0; k < my_tiles && !*abort_flag; ++k) {
        const ShtTcTile tl = tile_k(k);
        if (reject_tile(tl, abort_flag, a.err)) break;
        const TcGroup& G = a.g[tl.group];
        bool ok = true;
        for (int ks = 0; ks < tl.kst; ++ks) {
          if (!wait_bar(&pp.raw_empty[stage], phase ^ 1, pp, a.err, 9)) {
            ok = false;
            break;
          }
          // Rows r0 .. r0+127 as four 32-row boxes, contraction rows
          // d_row + ks*BK .. +BK-1.
          mbar_arrive_expect_tx(&pp.full_raw[stage], kRawStage);
          unsigned char* raw = sRaw + stage * kRawStage;
#pragma unroll
          for (int q = 0; q < BM / 32; ++q)
            tma_load_2d(raw + q * kRawBox, &G.data_map, tl.r0 + 32 * q,
                        (int)(tl.d_row + (int64_t)ks * BK), &pp.full_raw[stage]);
          armed[stage] = (int)phase;
          if (++stage == S) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
      }
      // Drain: every armed copy lands before the CTA exits (after an abort
      // this wait keeps a late copy from writing freed shared memory).
      for (int s = 0; s < S; ++s) {
        long long t0 = clock64();
        if (armed[s] >= 0)
          while (!mbar_try_wait(&pp.full_raw[s], (uint32_t)armed[s]) && clock64() - t0 < kWaitBudget) {
          }
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------------- MMA
    if (lane == 0) {
      int stage = 0;  // shared stage (table; data when !A_TMEM)
      uint32_t phase = 0;
      int aslot = 0;  // TMEM data slot (A_TMEM)
      uint32_t aphase = 0;
      uint32_t acc_it = 0;  // accumulator set = acc_it % NBUF, parity = (acc_it / NBUF) & 1
      bool issued = false;
      for (int k = 0; k < my_tiles && !*abort_flag; ++k) {
        const ShtTcTile tl = tile_k(k);
        if (reject_tile(tl, abort_flag, a.err)) break;
        if (tl.kst == 0) continue;
        const uint32_t buf = acc_it % NBUF, acc_phase = (acc_it / NBUF) & 1;
        if (!wait_bar(&pp.acc_empty[buf], acc_phase ^ 1, pp, a.err, 2)) break;
        const uint32_t d_set = tmem_base + buf * kAccCols;
        const uint32_t d_corr = d_set + NMAIN * NMAX;
        tc_fence_after();
        // A from TMEM is K-major (no transpose bit).
        const uint32_t idesc = Acc::A_TMEM ? instr_desc(tl.nsize) & ~(1u << 15) : instr_desc(tl.nsize);
        const uint32_t lbo_b = (uint32_t)tl.nsize * 16;
        const int nsteps = tl.kst * (BK / 16);  // K steps of 16 in the tile
        // Segment of step k: floor(k * NMAIN / nsteps), advanced at the
        // boundaries ceil(s * nsteps / NMAIN) instead of divided per step.
        int seg = 0, seg_prev = -1;
        int next_b = NMAIN > 1 ? (nsteps + NMAIN - 1) / NMAIN : nsteps;
        bool ok = true;
        for (int ks = 0; ks < tl.kst; ++ks) {
          if (!wait_fast(Acc::A_TMEM ? &pp.full_a[aslot] : &pp.full_a[stage],
                         Acc::A_TMEM ? aphase : phase, pp, a.err, 3) ||
              !wait_fast(&pp.full_b[stage], phase, pp, a.err, 4)) {
            ok = false;
            break;
          }
          tc_fence_after();
          // Descriptors of the stage's operands; a K step of 16 (two K groups
          // of 8) advances the start-address field by 2 LBO / 16.
          const uint64_t da0 = smem_desc(smem_u32(sA + stage * NPARTS * kAPart), kALbo, 128);
          const uint64_t db0 = smem_desc(smem_u32(sB + stage * NPARTS * kBPart), lbo_b, 128);
#pragma unroll
          for (int j = 0; j < BK / 16; ++j) {
            const uint64_t da1 = da0 + (uint64_t)(j * 2 * kALbo / 16);
            const uint64_t da2 = da1 + (uint64_t)(kAPart / 16);
            const uint64_t db1 = db0 + (uint64_t)(j * 2 * lbo_b / 16);
            const uint64_t db2 = db1 + (uint64_t)(kBPart / 16);
            const int step = ks * (BK / 16) + j;
            if (step >= next_b && seg < NMAIN - 1) {  // contiguous thirds of the K steps
              ++seg;
              next_b = ((seg + 1) * nsteps + NMAIN - 1) / NMAIN;
            }
            const uint32_t accum_main = seg == seg_prev ? 1u : 0u;
            seg_prev = seg;
            const uint32_t accum_corr = step > 0 ? 1u : 0u;
            if constexpr (Acc::A_TMEM) {
              const uint32_t ta1 = tmem_base + (uint32_t)(Acc::kATmem + aslot * 32 + j * 8);
              const uint32_t ta2 = ta1 + 16;
              mma_f16_ts(d_set + (uint32_t)(seg * NMAX), ta1, db1, idesc, accum_main);  // a1 b1
              mma_f16_ts(d_corr, ta1, db2, idesc, accum_corr);                              // a1 b2
              mma_f16_ts(d_corr, ta2, db1, idesc, 1u);                                      // a2 b1
            } else {
              mma_f16(d_set + (uint32_t)(seg * NMAX), da1, db1, idesc, accum_main);  // a1 b1
              mma_f16(d_corr, da1, db2, idesc, accum_corr);                              // a1 b2
              mma_f16(d_corr, da2, db1, idesc, 1u);                                      // a2 b1
            }
          }
          issued = true;
          mma_commit(&pp.empty[stage]);  // frees the stage when these MMAs finish
          if (++stage == S) { stage = 0; phase ^= 1; }
          if constexpr (Acc::A_TMEM) {
            mma_commit(&pp.a_empty[aslot]);  // and the TMEM data slot
            if (++aslot == NA) { aslot = 0; aphase ^= 1; }
          }
        }
        if (!ok) break;
        mma_commit(&pp.acc_full[buf]);
        ++acc_it;
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
    // Per tile: TMEM -> registers -> scaled values stored straight to global
    // memory.  Thread `row` of a warp pair owns one data row r of the tile and
    // half of its columns; for each column the warp's 32 lanes write 32
    // consecutive r (one 128-byte line per store), so no staging through
    // shared memory is needed (the tensor core's operand reads have its whole
    // bandwidth).  The accumulator goes back to the MMA warp once its last
    // chunk is in registers.  Every decision that steers the epilogue's named barrier is reduced over
    // its eight warps (epi_bar_or), so all 256 threads take the same path,
    // and the warp-collective tcgen05.ld is entered warp-uniformly.
    const int eg = warp & 3;  // TMEM lane group accessible to this warp
    const int half = (warp - kEpiWarp0) / 4;
    const int row = eg * 32 + lane;
    float* cs_s = reinterpret_cast<float*>(smem + Acc::kOffCs) + (warp - kEpiWarp0) * NMAX;  // this warp's copy
    uint32_t acc_it = 0;
    for (int k = 0; k < my_tiles; ++k) {
      const ShtTcTile tl = tile_k(k);
      if (reject_tile(tl, abort_flag, a.err)) break;  // the same tile for all 256 threads
      const TcGroup& G = a.g[tl.group];
      const int64_t R = G.R;
      const int64_t r = tl.r0 + row;
      float* outb = G.out + tl.c_row * R;
      const int cbeg = half * (NMAX / 2), cend = min(tl.nsize, cbeg + NMAX / 2);
      if (tl.kst == 0) {
        // empty contraction (K = 0): the output block is zero
        if (r < R)
          for (int x = tl.n0 + cbeg; x < min(tl.n0 + cend, tl.X); ++x) outb[(int64_t)x * R + r] = 0.f;
        continue;
      }
      // The tile's row and column scales are fetched while the MMAs run: the
      // column scales into this warp's shared copy (one L2 round trip per
      // tile instead of one per 16-column chunk).
      const float rs = r < R ? __frcp_rn(row_scale(G, r)) : 0.f;  // exact: a power of two
      {
        const float* cs = G.colscale + tl.cs;
        __syncwarp();  // the previous tile's reads of cs_s are done
#pragma unroll
        for (int j = 0; j < NMAX / 32; ++j) {
          const int c = j * 32 + lane;
          cs_s[c] = (c < tl.nsize && tl.n0 + c < tl.X) ? cs[tl.n0 + c] : 0.f;
        }
        __syncwarp();
      }
      const uint32_t buf = acc_it % NBUF, acc_phase = (acc_it / NBUF) & 1;
      const bool failed = !wait_bar(&pp.acc_full[buf], acc_phase, pp, a.err, 5);
      if (epi_bar_or(failed)) break;
      tc_fence_after();
      const uint32_t lane_off = ((uint32_t)(eg * 32) << 16) + buf * kAccCols;
      // A tile with fewer K steps than NMAIN leaves the last main
      // accumulators unwritten: only the segments that exist are read.
      const int nsteps = tl.kst * (BK / 16);
      const int nseg = nsteps < NMAIN ? nsteps : NMAIN;
      // Columns past the problem's extent are not stored.
      const int ncols = min(tl.nsize, tl.X - tl.n0);
      float* dst = outb + (int64_t)tl.n0 * R + r;
      bool released = false;
      for (int c0 = cbeg; c0 < cend; c0 += 16) {
        // The corrections and the first main segment, then the other
        // segments one at a time: the sum is formed in the order corrections
        // + segment 0 + segment 1 + ..., with at most 32 registers of
        // accumulator data live.
        float acc[16];
        {
          uint32_t rc[16], rm[16];
          tmem_ld16_async(tmem_base + lane_off + (uint32_t)(NMAIN * NMAX + c0), rc);
          tmem_ld16_async(tmem_base + lane_off + (uint32_t)c0, rm);
          tmem_wait16<true>(rc);
          tmem_wait16<false>(rm);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = __uint_as_float(rc[i]) + __uint_as_float(rm[i]);
        }
#pragma unroll
        for (int g = 1; g < NMAIN; ++g) {
          if (g < nseg) {
            uint32_t rm[16];
            tmem_ld16_async(tmem_base + lane_off + (uint32_t)(g * NMAX + c0), rm);
            tmem_wait16<true>(rm);
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] += __uint_as_float(rm[i]);
          }
        }
        if (c0 + 16 >= cend) {
          // The last chunk is in registers: the accumulator set is free.
          tc_fence_before();
          mbar_arrive(&pp.acc_empty[buf]);
          released = true;
        }
        if (r < R) {
          // 32-bit column offsets (R < 2^26 is checked at launch): a 64-bit
          // address per store would hold 32 more registers.
          float* col = dst + (int64_t)c0 * R;
          const int r32 = (int)R;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const float4 c4 = *reinterpret_cast<const float4*>(cs_s + c0 + 4 * q);
            const float cq[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int i4 = 0; i4 < 4; ++i4) {
              const int i = 4 * q + i4;
              if (c0 + i < ncols) col[i * r32] = acc[i] * rs * cq[i4];
            }
          }
        }
      }
      if (!released) {  // no columns in this warp's half
        tc_fence_before();
        mbar_arrive(&pp.acc_empty[buf]);
      }
      ++acc_it;
    }
  } else if constexpr (Acc::A_TMEM) {
    // ------------------------------------------- converters (A into TMEM)
    // Warp -> TMEM lane quarter q4 = warp % 4 (the lanes it may access) and
    // K half kh; lane -> data row q4*32 + lane of the tile.  Each thread
    // splits its row's 16 K values of the stage into FP16 hi/lo pairs and
    // stores them as 8 + 8 columns of the stage's A slot.
    const int q4 = warp & 3, kh = (warp - kConvWarp0) >> 2;
    const int rowi = q4 * 32 + lane;
    const uint32_t lane_base = tmem_base + ((uint32_t)(q4 * 32) << 16);
    int stage = 0;  // raw stage of the data (TMA)
    uint32_t phase = 0;
    int aslot = 0;  // TMEM data slot
    uint32_t aphase = 0;
    for (int k = 0; k < my_tiles; ++k) {
      const ShtTcTile tl = tile_k(k);
      if (reject_tile(tl, abort_flag, a.err)) break;
      if (tl.kst == 0) continue;
      const TcGroup& G = a.g[tl.group];
      const int64_t R = G.R;
      const int64_t r = tl.r0 + rowi;
      const float sc = r < R ? row_scale(G, r) : 1.f;
      const float* Db = G.data + tl.d_row * R;
      bool ok = true;
      for (int ks = 0; ks < tl.kst; ++ks) {
        float v[16];
        if (G.use_tma) {
          // Box q4 of the stage holds rows q4*32 .. +31 as 128-byte k rows,
          // 16-byte chunks swizzled by k % 8.
          ok = wait_bar(&pp.full_raw[stage], phase, pp, a.err, 8);
          if (!ok) break;
          const unsigned char* box = sRaw + stage * kRawStage + q4 * kRawBox;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int kl = kh * 16 + i;
            const float x = *reinterpret_cast<const float*>(
                box + kl * 128 + ((((lane >> 2) ^ (kl & 7))) << 4) + (lane & 3) * 4);
            v[i] = ks * BK + kl < tl.K ? x : 0.f;  // rows past K belong to the next problem
          }
          __syncwarp();  // the warp's reads of the raw stage are done
          if (lane == 0) mbar_arrive(&pp.raw_empty[stage]);
          if (++stage == S) { stage = 0; phase ^= 1; }
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int k = ks * BK + kh * 16 + i;
            v[i] = (k < tl.K && r < R) ? __ldg(Db + (int64_t)k * R + r) : 0.f;
          }
        }
        // The TMEM slot's previous MMAs are done.
        ok = wait_bar(&pp.a_empty[aslot], aphase ^ 1, pp, a.err, 7);
        if (!ok) break;
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float x0 = v[2 * c] * sc, x1 = v[2 * c + 1] * sc;
          const float a0 = round_to_11_bits(x0), a1 = round_to_11_bits(x1);
          const __half2 h1 = __floats2half2_rn(a0, a1);           // exact: 11 significant bits
          const __half2 h2 = __floats2half2_rn(x0 - a0, x1 - a1);  // the remainder, exact in FP32
          hi[c] = *reinterpret_cast<const uint32_t*>(&h1);
          lo[c] = *reinterpret_cast<const uint32_t*>(&h2);
        }
        const uint32_t ta = lane_base + (uint32_t)(Acc::kATmem + aslot * 32 + kh * 8);
        tmem_st8(ta, hi);
        tmem_st8(ta + 16, lo);
        tmem_wait_st();
        tc_fence_before();
        mbar_arrive(&pp.full_a[aslot]);
        if (++aslot == NA) { aslot = 0; aphase ^= 1; }
      }
      if (!ok) break;
    }
  } else {
    // --------------------------------------------------------- converters
    // Thread -> (kk = ct % 8, 8-row group mg = (ct/8) % 16), K groups
    // kg = ct/128 + 2j (j < BK/16): each store is one 16-byte core-matrix row,
    // and a warp's 32 stores cover 512 contiguous bytes (no bank conflicts).
    const int ct = threadIdx.x - kConvWarp0 * 32;  // 0..255
    const int kk = ct & 7, mg = (ct >> 3) & 15, kgs = ct >> 7;
    int stage = 0;  // converted-operand stage (shared with the table stage and the MMA)
    uint32_t phase = 0;
    int rstage = 0;  // raw stage of the data (TMA)
    uint32_t rphase = 0;
    for (int k = 0; k < my_tiles; ++k) {
      const ShtTcTile tl = tile_k(k);
      if (reject_tile(tl, abort_flag, a.err)) break;
      if (tl.kst == 0) continue;
      const TcGroup& G = a.g[tl.group];
      const int64_t R = G.R;
      const float* Db = G.data + tl.d_row * R;
      const int64_t rbase = tl.r0 + mg * 8;
      float sc[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) sc[i] = rbase + i < R ? row_scale(G, rbase + i) : 1.f;
      const bool full_rows = rbase + 8 <= R && (R % 4) == 0;
      // Stage ks + 1 is loaded while stage ks waits for its slot and is
      // converted (two register buffers, swapped by a 2x unrolled loop).
      auto load_stage = [&](int ks, float (&v)[BK / 16][8]) {
#pragma unroll
        for (int j = 0; j < BK / 16; ++j) {
          const int k = ks * BK + (kgs + 2 * j) * 8 + kk;
          if (k < tl.K) {
            const float* p = Db + (int64_t)k * R + rbase;
            if (full_rows) {
              const float4 u0 = __ldg(reinterpret_cast<const float4*>(p));
              const float4 u1 = __ldg(reinterpret_cast<const float4*>(p + 4));
              v[j][0] = u0.x; v[j][1] = u0.y; v[j][2] = u0.z; v[j][3] = u0.w;
              v[j][4] = u1.x; v[j][5] = u1.y; v[j][6] = u1.z; v[j][7] = u1.w;
            } else {
#pragma unroll
              for (int i = 0; i < 8; ++i) v[j][i] = (rbase + i < R) ? __ldg(p + i) : 0.f;
            }
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) v[j][i] = 0.f;
          }
        }
      };
      // The stage's data from the TMA-filled shared tile: boxes of 32 rows
      // x 32 k with the 16-byte chunks of each 128-byte k row XOR-swizzled
      // by (k mod 8), which makes this warp's reads (8 consecutive k of one
      // 8-row group per quarter warp) bank-conflict free.
      auto fetch_raw = [&](int ks, float (&v)[BK / 16][8]) {
        const unsigned char* raw = sRaw + rstage * kRawStage + (mg >> 2) * kRawBox;
#pragma unroll
        for (int j = 0; j < BK / 16; ++j) {
          const int kl = (kgs + 2 * j) * 8 + kk;  // k within the stage
          const unsigned char* row = raw + kl * 128;
          const int c0 = (mg & 3) * 2;
          const float4 u0 = *reinterpret_cast<const float4*>(row + ((c0 ^ (kl & 7)) << 4));
          const float4 u1 = *reinterpret_cast<const float4*>(row + (((c0 + 1) ^ (kl & 7)) << 4));
          const bool live = ks * BK + kl < tl.K;  // rows past K belong to the next problem
          v[j][0] = live ? u0.x : 0.f; v[j][1] = live ? u0.y : 0.f;
          v[j][2] = live ? u0.z : 0.f; v[j][3] = live ? u0.w : 0.f;
          v[j][4] = live ? u1.x : 0.f; v[j][5] = live ? u1.y : 0.f;
          v[j][6] = live ? u1.z : 0.f; v[j][7] = live ? u1.w : 0.f;
        }
      };
      auto convert_stage = [&](const float (&v)[BK / 16][8], bool wait_slot) -> bool {
        if (wait_slot && !wait_bar(&pp.empty[stage], phase ^ 1, pp, a.err, 7)) return false;
        unsigned char* dst = sA + stage * NPARTS * kAPart;
#pragma unroll
        for (int j = 0; j < BK / 16; ++j) {
          const int kg = kgs + 2 * j;
          __align__(16) __half2 h1[4];
          __align__(16) __half2 h2[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float x0 = v[j][2 * i] * sc[2 * i], x1 = v[j][2 * i + 1] * sc[2 * i + 1];
            const float a0 = round_to_11_bits(x0), a1 = round_to_11_bits(x1);
            h1[i] = __floats2half2_rn(a0, a1);           // exact: 11 significant bits
            h2[i] = __floats2half2_rn(x0 - a0, x1 - a1);  // the remainder, exact in FP32
          }
          const int off = kg * kALbo + mg * 128 + kk * 16;
          *reinterpret_cast<uint4*>(dst + off) = *reinterpret_cast<const uint4*>(h1);
          *reinterpret_cast<uint4*>(dst + kAPart + off) = *reinterpret_cast<const uint4*>(h2);
        }
        fence_proxy_async();
        mbar_arrive(&pp.full_a[stage]);
        if (++stage == S) { stage = 0; phase ^= 1; }
        return true;
      };
      bool ok = true;
      float va[BK / 16][8], vb[BK / 16][8];
      if (G.use_tma) {
        // Read the raw stage into registers and hand it back at once, then
        // wait for the converted-operand slot.
        for (int ks = 0; ks < tl.kst && ok; ++ks) {
          ok = wait_bar(&pp.full_raw[rstage], rphase, pp, a.err, 8);
          if (!ok) break;
          fetch_raw(ks, va);
          __syncwarp();  // the warp's reads of the raw stage are done
          if ((threadIdx.x & 31) == 0) mbar_arrive(&pp.raw_empty[rstage]);
          if (++rstage == S) { rstage = 0; rphase ^= 1; }
          ok = convert_stage(va, true);
        }
      } else {
        load_stage(0, va);
        for (int ks = 0; ks < tl.kst && ok; ks += 2) {
          if (ks + 1 < tl.kst) load_stage(ks + 1, vb);
          ok = convert_stage(va, true);
          if (!ok || ks + 1 >= tl.kst) break;
          if (ks + 2 < tl.kst) load_stage(ks + 2, va);
          ok = convert_stage(vb, true);
        }
      }
      if (!ok) break;
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
// [k-stage][part 2][kg BK/8][ng nsize/8][kk 8][nn 8] halves, the parts being
// the two FP16 terms (hi, lo) of the scaled FP64 value.
__global__ void image_kernel(ImgArgs a, const BlockInfo* blocks, int nblocks, unsigned char* img) {
  const int b = blockIdx.y;
  if (b >= nblocks) return;
  const BlockInfo bi = blocks[b];
  const ShtGemmDesc d = a.descs[bi.problem];
  const int64_t per_part = (int64_t)bi.nsize * BK;  // halves per part per stage
  const int64_t total = per_part * bi.kst;
  __half* base = reinterpret_cast<__half*>(img + bi.off);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int ks = (int)(e / per_part);
    int rem = (int)(e % per_part);
    const int nn = rem & 7;
    rem >>= 3;
    const int kk = rem & 7;
    rem >>= 3;
    const int ng = rem % (bi.nsize / 8);
    const int kg = rem / (bi.nsize / 8);
    const int x = bi.n0 + ng * 8 + nn;
    const int k = ks * BK + kg * 8 + kk;
    __half p1 = __float2half_rn(0.f), p2 = p1;
    if (x < d.X && k < d.K) {
      const double v = a.tab[d.t_off + (int64_t)k * d.ldt + x] * (double)a.colmul[a.cs_off[bi.problem] + x];
      p1 = __float2half_rn((float)v);
      p2 = __float2half_rn((float)(v - (double)__half2float(p1)));
    }
    const int64_t pos = ((int64_t)(kg * (bi.nsize / 8) + ng) * 8 + kk) * 8 + nn;
    __half* st = base + (int64_t)ks * NPARTS * per_part;
    st[pos] = p1;
    st[per_part + pos] = p2;
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
  tc->tiles = tc_cache_create();
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
          off += (int64_t)kst * NPARTS * ns * BK * 2;
        }
      }
      tc->img_bytes[dir] = off;
      tc->cs_elems[dir] = cso;
      SHT_CUDA_OR_THROW(cudaMalloc(&tc->d_img_off[dir], 8 * std::max<size_t>(tc->img_off[dir].size(), 1)));
      upload_now(tc->d_img_off[dir], tc->img_off[dir].data(), 8 * tc->img_off[dir].size());
      SHT_CUDA_OR_THROW(cudaMalloc(&tc->d_cs_off[dir], 8 * np));
      upload_now(tc->d_cs_off[dir], tc->cs_off[dir].data(), 8 * np);
    }
    ShtGemmDesc* dd[2];
    BlockInfo* db[2];
    float* colmul[2];
    for (int dir = 0; dir < 2; ++dir) {
      SHT_CUDA_OR_THROW(cudaMalloc(&dd[dir], sizeof(ShtGemmDesc) * d64[dir].size()));
      upload_now(dd[dir], d64[dir].data(), sizeof(ShtGemmDesc) * d64[dir].size());
      SHT_CUDA_OR_THROW(cudaMalloc(&db[dir], sizeof(BlockInfo) * std::max<size_t>(blocks[dir].size(), 1)));
      upload_now(db[dir], blocks[dir].data(), sizeof(BlockInfo) * blocks[dir].size());
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
    SHT_CUDA_OR_THROW(cudaFuncSetAttribute(tc_gemm_kernel<kOverlapped>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kOverlapped::kSmemBytes));
    SHT_CUDA_OR_THROW(cudaFuncSetAttribute(tc_gemm_kernel<kAccurate>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kAccurate::kSmemBytes));
    SHT_CUDA_OR_THROW(cudaFuncSetAttribute(tc_gemm_kernel<kTmemA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kTmemA::kSmemBytes));
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
  }
  tc_cache_destroy(tc->tiles);
  delete tc;
  p->tc = nullptr;
}

int64_t tc_table_bytes(const sht_plan* p, int kind) {
  const ShtTc16* tc = p->tc;
  if (!tc || kind < 0 || kind >= 5) return 0;
  const int dir = kind == 0 || kind == 1 ? 0 : 1;
  return tc->img_bytes[dir] + 4 * tc->cs_elems[dir];
}

struct TcTileCache {
  struct List {
    ShtTcTile* d = nullptr;
    int n = 0;
  };
  // Key: per group (direction, R).  Lists live as long as the cache, so a
  // launch recorded in a CUDA graph keeps pointing at a live list.
  std::map<std::vector<int64_t>, List> lists;
  // Tensor maps of data operands, by (address, R, rows).
  std::map<std::vector<int64_t>, CUtensorMap> maps;
  std::mutex mu;
};

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      ptr = nullptr;
    return reinterpret_cast<EncodeTiledFn>(ptr);
  }();
  return fn;
}

// The data operand of a launch as a 2D FP32 tensor [rows][R] (R innermost),
// read in 32 x 32 boxes with the 128-byte swizzle the converters undo.
// Requires R % 4 == 0 (16-byte row pitch); false if it cannot be encoded.
bool data_map(TcTileCache* c, const float* data, int64_t R, int64_t rows, CUtensorMap* out) {
  if (R % 4 != 0 || R <= 0 || rows <= 0) return false;
  std::vector<int64_t> key{(int64_t)(uintptr_t)data, R, rows};
  auto it = c->maps.find(key);
  if (it != c->maps.end()) {
    *out = it->second;
    return true;
  }
  EncodeTiledFn fn = encode_tiled();
  if (fn == nullptr) return false;
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)R, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)R * 4};
  const cuuint32_t box[2] = {32, (cuuint32_t)BK};
  const cuuint32_t elem[2] = {1, 1};
  if (fn(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(data), dims, strides, box,
         elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  c->maps.emplace(key, m);
  *out = m;
  return true;
}

}  // namespace

TcTileCache* tc_cache_create() { return new TcTileCache(); }

void tc_cache_destroy(TcTileCache* c) {
  if (!c) return;
  for (auto& e : c->lists) cudaFree(e.second.d);
  delete c;
}

TcTileCache* tc_plan_cache(const sht_plan* p) { return p->tc ? p->tc->tiles : nullptr; }

void launch_gemm_tc_groups(const TcGroupSpec* g, int ngroups, TcTileCache* cache, cudaStream_t s) {
  SHT_REQUIRE(ngroups >= 1 && ngroups <= kMaxTcGroups, "tensor-core launch: 1 to 4 groups");
  SHT_REQUIRE(cache != nullptr, "tensor-core launch: no tile cache");
  const int order = g[0].plan->tune_tile_order;
  std::vector<int64_t> key{order};
  int64_t rows = 0;
  for (int i = 0; i < ngroups; ++i) {
    SHT_REQUIRE(g[i].plan->tc != nullptr, "tensor-core tables not built");
    SHT_REQUIRE(g[i].R < ((int64_t)1 << 26), "tensor-core launch: too many data rows");
    // Plans of one cache differ in their descriptors: the key names the plan.
    key.push_back((int64_t)(uintptr_t)g[i].plan);
    key.push_back(g[i].direction);
    key.push_back(g[i].flip);
    key.push_back(g[i].R);
    rows += g[i].R;
  }
  if (rows == 0) return;
  TcTileCache::List list;
  {
    std::lock_guard<std::mutex> lock(cache->mu);
    auto found = cache->lists.find(key);
    if (found == cache->lists.end()) {
      // Tiles: every (group, problem, n-tile) x every 128-row block, merged
      // over the groups and sorted by descending cost.
      std::vector<std::pair<int64_t, ShtTcTile>> v;
      for (int gi = 0; gi < ngroups; ++gi) {
        const sht_plan* p = g[gi].plan;
        const ShtTc16* tc = p->tc;
        const int dir = g[gi].direction;
        const int np = (int)tc->nt_of[dir].size();
        for (int i = 0; i < np; ++i) {
          const int nt = tc->nt_of[dir][i], ns = tc->nsize_of[dir][i], kst = tc->kst_of[dir][i];
          if (p->h_desc[dir][0][i].X == 0) continue;
          const ShtGemmDesc& d = p->h_desc[dir][g[gi].flip][i];
          // Order 0: a column tile's row blocks are adjacent (they share its
          // table image); order 1: a row block's column tiles are adjacent
          // (they share its converted data rows).
          const int64_t nr = div_up(g[gi].R, BM);
          for (int64_t o = 0; o < nt * nr; ++o) {
            const int j = order == 0 ? (int)(o / nr) : (int)(o % nt);
            const int64_t r0 = BM * (order == 0 ? o % nr : o / nt);
            ShtTcTile t{};
            t.group = gi;
            t.problem = i;
            t.n0 = j * ns;
            t.nsize = ns;
            t.kst = kst;
            t.r0 = (int)r0;
            t.X = d.X;
            t.K = d.K;
            t.img = tc->img_off[dir][tc->img_base[dir][i] + j];
            t.d_row = d.d_row;
            t.c_row = d.c_row;
            t.cs = tc->cs_off[dir][i];
            v.push_back({(int64_t)ns * kst * BK + 4096, t});
          }
        }
      }
      std::stable_sort(v.begin(), v.end(),
                       [](const auto& a, const auto& b) { return a.first > b.first; });
      std::vector<ShtTcTile> flat;
      flat.reserve(v.size());
      for (auto& e : v) flat.push_back(e.second);
      TcTileCache::List fresh;
      SHT_CUDA_OR_THROW(cudaMalloc(&fresh.d, sizeof(ShtTcTile) * std::max<size_t>(flat.size(), 1)));
      // The launch below may be on a non-blocking stream: the list must be on
      // the device before it is read (upload_now).
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      SHT_CUDA_OR_THROW(cudaStreamIsCapturing(s, &cap));
      SHT_REQUIRE(cap == cudaStreamCaptureStatusNone,
                  "tensor-core tile list built during stream capture: run the call once before "
                  "capturing it");
      upload_now(fresh.d, flat.data(), sizeof(ShtTcTile) * flat.size());
      fresh.n = (int)flat.size();
      found = cache->lists.emplace(key, fresh).first;
    }
    list = found->second;
  }
  if (list.n == 0) return;
  TcArgs a{};
  // All groups of a launch take the data by TMA, or none does (the loader
  // and the converters then agree on which barriers a stage completes).
  bool tma = true;
  {
    std::lock_guard<std::mutex> lock(cache->mu);
    for (int gi = 0; gi < ngroups && tma; ++gi) {
      const sht_plan* p = g[gi].plan;
      const int64_t rows = g[gi].direction == 0 ? p->cf_rows : (int64_t)(p->T + 1) * 2 * p->H;
      tma = data_map(cache, g[gi].data, g[gi].R, rows, &a.g[gi].data_map);
    }
  }
  int rs_off = 0;
  for (int gi = 0; gi < ngroups; ++gi) {
    const sht_plan* p = g[gi].plan;
    const ShtTc16* tc = p->tc;
    TcGroup& G = a.g[gi];
    G.use_tma = tma ? 1 : 0;
    G.img = (const unsigned char*)tc->img[g[gi].table_kind];
    G.colscale = tc->colscale[g[gi].table_kind];
    G.data = g[gi].data;
    G.rowmax = g[gi].rowmax;
    G.out = g[gi].out;
    G.R = g[gi].R;
    G.rs_off = rs_off;
    rs_off += (int)std::min<int64_t>(g[gi].R, kMaxRowScales + 1);
  }
  a.stage_rs = rs_off <= kMaxRowScales ? 1 : 0;
  a.rs_total = rs_off;
  a.tiles = list.d;
  a.n_tiles = list.n;
  a.err = g[0].plan->d_err;
  const int ctas = g[0].plan->tune_tc_ctas > 0 ? g[0].plan->tune_tc_ctas : g[0].plan->tc->sm_count;
  const int grid = std::min(list.n, ctas);
  if (g[0].plan->tune_accumulators == 1)
    tc_gemm_kernel<kOverlapped><<<grid, kThreads, kOverlapped::kSmemBytes, s>>>(a);
  else if (g[0].plan->tune_accumulators == 2)
    tc_gemm_kernel<kTmemA><<<grid, kThreads, kTmemA::kSmemBytes, s>>>(a);
  else
    tc_gemm_kernel<kAccurate><<<grid, kThreads, kAccurate::kSmemBytes, s>>>(a);
  SHT_CUDA_OR_THROW(cudaGetLastError());
}

void launch_gemm_tc(const sht_plan* p, int direction, int flip, int table_kind, const float* data,
                    const float* rowmax, float* out, int64_t R, cudaStream_t s) {
  SHT_REQUIRE(p->tc != nullptr, "tensor-core tables not built");
  TcGroupSpec g{p, direction, flip, table_kind, data, rowmax, out, R};
  launch_gemm_tc_groups(&g, 1, p->tc->tiles, s);
}

}  // namespace sht
