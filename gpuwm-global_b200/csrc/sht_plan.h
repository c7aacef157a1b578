// Internal plan object and the per-(order, parity) bookkeeping shared by the
// kernels.  Not part of the public ABI.
#pragma once

#include "sht_common.cuh"

// One (order m, degree-parity q) block of a Legendre contraction, the unit of
// work of every GEMM launch.  Offsets are element offsets into the table and
// ROW offsets into the data/output (multiplied by the call's row count R in
// the kernel).  C[x][r] = sum_k Tab[k][x] * D[k][r].
struct ShtGemmDesc {
  int64_t t_off;  // element offset of the table block
  int64_t d_row;  // row offset of the data block (k = 0)
  int64_t c_row;  // row offset of the output block (x = 0)
  int X;          // output extent (x)
  int K;          // contraction extent (k)
  int ldt;        // table leading dimension (padded x extent)
  int m;          // order (for epilogues)
};

// A tile of a GEMM launch: problem index and first x.
struct ShtGemmItem {
  int problem;
  int x0;
};

struct ShtTc16;  // split-precision tensor-core tables (sht_gemm_tc.cu)

struct sht_plan {
  int T = 0, nlat = 0, nlon = 0, H = 0, L = 0, prec = 0;
  int Hx = 0;         // H padded to a multiple of 4 (synthesis tables)
  bool nlat_odd = false;
  double radius = 0;
  int device = 0;
  bool geometry_only = false;

  // FP64 geometry on the device and a host copy.
  double* d_mu = nullptr;
  double* d_w = nullptr;
  double* d_coslat = nullptr;
  std::vector<double> h_mu, h_w, h_coslat;

  // Per (m, q) bookkeeping, index m*2+q.
  std::vector<int> e, ex;                        // count and padded count
  std::vector<int64_t> syn_off, ana_off, cf_row;  // table offsets, Cfold row offsets
  int64_t syn_total = 0, ana_total = 0, cf_rows = 0;

  // Tables in the plan's element type (double for F64, float otherwise).
  // Synthesis layout [m][q][i][h] (ld Hx); analysis layout [m][q][h][i] (ld ex).
  void* basis = nullptr;     // P_nm
  void* dbasis = nullptr;    // dP_nm / dphi
  void* analysis = nullptr;  // Gram-corrected 2 pi w P
  void* rot = nullptr;       // 2 pi w P / (a cos phi)
  void* shear = nullptr;     // 2 pi w dP / a

  ShtTc16* tc = nullptr;     // SPLIT16 tiles

  // FFT: twiddles exp(-2 pi i k / L), k < L, and exp(-2 pi i k / N), k <= L.
  void* tw_l = nullptr;
  void* tw_n = nullptr;
  std::vector<int> radices;
  int* d_radices = nullptr;
  bool fast_fft = false;           // register-resident kernels (sht_fft_fast.cu)
  bool force_generic_fft = false;  // SHT_FLAG_GENERIC_FFT
  // Autotuner settings (sht_plan_set_tuning).
  int tune_contraction = 0;  // 1: FP32 SIMT contraction on a split16 plan
  int tune_tile_order = 0;   // tensor-core tile order (0: row blocks innermost, 1: column tiles)
  int tune_tc_ctas = 0;      // tensor-core CTAs per launch (0: one per SM)
  int tune_simt_tile = 0;    // FP32 SIMT column tile (0: 128 wide; 1: 64 wide)
  int tune_accumulators = 0; // tensor-core accumulators (0: three K segments; 1: one, double-buffered;
                             // 2: two K segments, data operand in TMEM)

  // GEMM descriptors: [direction][flip] (direction 0 synthesis, 1 analysis).
  ShtGemmDesc* d_desc[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  std::vector<ShtGemmDesc> h_desc[2][2];
  ShtGemmItem* d_items[2] = {nullptr, nullptr};
  int n_items[2] = {0, 0};
  ShtGemmItem* d_items_narrow[2] = {nullptr, nullptr};  // FP32: 64-wide column tiles
  int n_items_narrow[2] = {0, 0};
  int n_problems = 0;
  int gemm_bx = 0;  // x tile of the SIMT kernel the item lists were built for

  // Scratch (grown on demand): two waists and two Cfold buffers.
  void* wfold[2] = {nullptr, nullptr};
  void* cfold[2] = {nullptr, nullptr};
  float* rowmax = nullptr;   // per data row max |value| (split-precision row scales)
  int64_t scratch_rows = 0;  // R capacity (rows = 2 * planes * fields)

  unsigned* d_err = nullptr;
  cudaStream_t last_stream = nullptr;

  // Host-resident streaming (sht_*_host): copy-in, compute and copy-out
  // streams and kHostSlots device slots of (input, intermediate, output)
  // chunk buffers, created on first use.
  static constexpr int kHostSlots = 3;
  struct HostStream {
    cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
    cudaEvent_t h2d[kHostSlots] = {}, comp[kHostSlots] = {}, d2h[kHostSlots] = {};
    void* buf[kHostSlots][3] = {};  // [slot][input, intermediate, output]
    size_t cap[3] = {0, 0, 0};      // bytes per slot of each buffer
  } hs;

  // Per-kernel timing (sht_plan_set_timing / sht_plan_read_timing).
  struct TimingRec {
    int kind;
    cudaEvent_t start, stop;
  };
  bool timing = false;
  std::vector<TimingRec> timing_recs;
  std::vector<cudaEvent_t> event_pool;
  int64_t launches[SHT_KIND_COUNT] = {};
  int64_t timed[SHT_KIND_COUNT] = {};
  double ms[SHT_KIND_COUNT] = {};

  size_t elem() const { return prec == SHT_PREC_F64 ? 8 : 4; }
  int64_t wfold_elems(int64_t R) const { return int64_t(T + 1) * 2 * H * R; }
  int64_t cfold_elems(int64_t R) const { return cf_rows * R; }
};

namespace sht {

// Geometry and tables (sht_geometry.cu).
void build_geometry_and_tables(sht_plan* p, cudaStream_t s);

// FFT (sht_fft.cu).
void build_fft(sht_plan* p, cudaStream_t s);
// rowmax (optional): per data row r (plane/field/re-im), the running maximum
// of |value| over everything the kernel writes, merged with atomicMax on the
// float bits (the row scales of the split-precision contraction).
template <typename T>
void launch_forward_fold(const sht_plan* p, const T* g0, const T* g1, int64_t planes,
                         T* wfold, cudaStream_t s, float* rowmax = nullptr);
// Inverse modes.
enum UnfoldMode { kUnfoldScalar = 0, kUnfoldZonal = 1, kUnfoldGradient = 2, kUnfoldWind = 3,
                  kUnfoldMeridional = 4 };
template <typename T>
void launch_inverse_unfold(const sht_plan* p, int mode, const T* wP, const T* wD,
                           int64_t planes, T* out0, T* out1, cudaStream_t s);

// Register-resident FP32 FFTs for nlon = 64 F, F in {2,3,4,6,8,12,16,24}
// (sht_fft_fast.cu).
bool fast_fft_supported(const sht_plan* p);
void fast_fft_init_constants(cudaStream_t s);
void fast_forward_fold(const sht_plan* p, const float* g0, const float* g1, int64_t planes,
                       float* wfold, cudaStream_t s, float* rowmax = nullptr);
void fast_inverse_unfold(const sht_plan* p, int mode, const float* wP, const float* wD,
                         int64_t planes, float* out0, float* out1, cudaStream_t s);

// SIMT Legendre GEMM (sht_gemm_simt.cu).
void build_gemm_items(sht_plan* p);
template <typename T>
void launch_gemm_simt(const sht_plan* p, int direction, int flip, const T* table,
                      const T* data, T* out, int64_t R, cudaStream_t s);

// Pack / unpack / elementwise (sht_pack.cu).
enum PackMode { kPackPlain = 0, kPackInvLap = 1 };
template <typename T>
void launch_pack(const sht_plan* p, const T* coeff0, const T* coeff1, int64_t planes,
                 int mode, T* cfold, cudaStream_t s, float* rowmax = nullptr);

// Warp-level merge of per-thread row maxima: lanes with equal lane % nper
// hold the same column (complex index col); lanes < nper publish.
__device__ __forceinline__ void rowmax_merge(float* rowmax, int64_t col, bool valid, float mre,
                                             float mim, int nper) {
  const int lane = threadIdx.x & 31;
  for (int off = nper; off < 32; off <<= 1) {
    mre = fmaxf(mre, __shfl_xor_sync(0xffffffffu, mre, off));
    mim = fmaxf(mim, __shfl_xor_sync(0xffffffffu, mim, off));
  }
  if (lane < nper && valid) {
    atomicMax(reinterpret_cast<int*>(rowmax + 2 * col), __float_as_int(mre));
    atomicMax(reinterpret_cast<int*>(rowmax + 2 * col + 1), __float_as_int(mim));
  }
}
// kUnpackDiv: divergence alone, D = i m rot[u] - shear[v], from single-field
// rotational (cf0, u) and shear (cf1, v) outputs.
enum UnpackMode { kUnpackScalar = 0, kUnpackVorDiv = 1, kUnpackDiv = 2 };
template <typename T>
void launch_unpack(const sht_plan* p, int mode, const T* cf0, const T* cf1, int64_t planes,
                   T* out0, T* out1, cudaStream_t s);
enum ElemMode { kElemProject = 0, kElemLaplacian = 1, kElemInvLaplacian = 2 };
template <typename T>
void launch_elementwise(const sht_plan* p, int mode, const T* in, int64_t planes, T* out,
                        cudaStream_t s);

// Semi-implicit maps (sht_helmholtz.cu).  `mats` packs B, C, V, V^-1,
// lambda and, when has_thermo, W, W^-1, mu (the thermodynamic block's modes).
enum SemiMode { kSemiSolve = 0, kSemiApply = 1, kSemiHalf = 2, kSemiLinear = 3 };
template <typename T>
void launch_semi_implicit(const sht_plan* p, int nlev, const T* mats, bool has_thermo, int mode,
                          double dt, double alpha, const T* div, const T* theta, const T* lnps,
                          T* odiv, T* otheta, T* olnps, T* metric, T* cfold, float* rowmax,
                          cudaStream_t s);
template <typename T>
void launch_helmholtz(const sht_plan* p, int nlev, const T* mats, double tau_w,
                      const T* div, const T* theta, const T* lnps, T* odiv, T* otheta,
                      T* olnps, cudaStream_t s);

// Reference-layout Fourier waist <-> folded waist (sht_waist.cu).
template <typename T>
void launch_waist_export(const sht_plan* p, const T* wfold, int64_t planes, double c, int zonal,
                         T* waist, cudaStream_t s);
template <typename T>
void launch_waist_import(const sht_plan* p, const T* waist, int64_t planes, double c, T* wfold,
                         float* rowmax, cudaStream_t s, int fields = 1);

// Split-precision tensor-core path (sht_gemm_tc.cu).
void build_tc_tables(sht_plan* p, const double* basis64, const double* dbasis64,
                     const double* analysis64, const double* rot64, const double* shear64,
                     cudaStream_t s);
void destroy_tc_tables(sht_plan* p);
// Device bytes of one table kind's FP16 hi/lo image and column scales.
int64_t tc_table_bytes(const sht_plan* p, int kind);
void launch_gemm_tc(const sht_plan* p, int direction, int flip, int table_kind,
                    const float* data, const float* rowmax, float* out, int64_t R,
                    cudaStream_t s);

// Several contractions in one persistent tensor-core launch (the two tables
// of a gradient, wind or vordiv call; the plans of a batch).
constexpr int kMaxTcGroups = 4;
struct TcGroupSpec {
  const sht_plan* plan;
  int direction, flip, table_kind;
  const float* data;
  const float* rowmax;
  float* out;
  int64_t R;
};
struct TcTileCache;  // merged tile lists, keyed by the groups' (direction, R)
TcTileCache* tc_cache_create();
void tc_cache_destroy(TcTileCache* c);
TcTileCache* tc_plan_cache(const sht_plan* p);  // the plan's own tile lists
void launch_gemm_tc_groups(const TcGroupSpec* groups, int ngroups, TcTileCache* cache,
                           cudaStream_t s);

}  // namespace sht
