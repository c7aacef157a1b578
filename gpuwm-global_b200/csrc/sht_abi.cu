// C ABI of the b200sht library: plan lifecycle, scratch, and the transform
// entry points declared in include/b200sht.h.  Each entry point validates its
// arguments, enqueues kernels on the caller's stream and returns a status; a
// failure leaves a thread-local message (sht_last_error).
#include <cstdio>
#include <exception>
#include <mutex>

#include "sht_plan.h"

// Plans run together (sht_batch_create).  The batch borrows its plans; its
// own tile cache holds the merged tensor-core tile lists.
struct sht_batch {
  std::vector<sht_plan*> plans;
  std::vector<int64_t> planes;
  sht::TcTileCache* cache = nullptr;
};

// A vertical structure operator resident on the plan's device: B, C, the
// modal basis and its inverse, and the eigenvalues, packed in the plan's
// arithmetic type in the order launch_helmholtz reads them.
struct sht_vertical {
  int device = 0;
  int prec = 0;
  int nlev = 0;
  bool thermo = false;  // W, W^-1 and mu follow (half maps)
  void* mats = nullptr;
  void* metric = nullptr;  // one value of the plan's type: max |D' - D| of the last map
};

namespace sht {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }
void clear_error() { g_error.clear(); }

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

enum TableKind { kBasis = 0, kDBasis = 1, kAnalysis = 2, kRot = 3, kShear = 4 };

cudaEvent_t pool_event(sht_plan* p) {
  if (!p->event_pool.empty()) {
    cudaEvent_t e = p->event_pool.back();
    p->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  SHT_CUDA_OR_THROW(cudaEventCreate(&e));
  return e;
}

// Counts a launch of `kind` and, with timing on, brackets it with events.
class KernelScope {
 public:
  KernelScope(sht_plan* p, int kind, cudaStream_t s) : p_(p), kind_(kind), s_(s) {
    p_->launches[kind_]++;
    if (p_->timing) {
      start_ = pool_event(p_);
      SHT_CUDA_OR_THROW(cudaEventRecord(start_, s_));
    }
  }
  ~KernelScope() {
    if (start_ == nullptr) return;
    cudaEvent_t stop = nullptr;
    try {
      stop = pool_event(p_);
    } catch (...) {
      return;
    }
    if (cudaEventRecord(stop, s_) == cudaSuccess) p_->timing_recs.push_back({kind_, start_, stop});
  }

 private:
  sht_plan* p_;
  int kind_;
  cudaStream_t s_;
  cudaEvent_t start_ = nullptr;
};

const void* table_ptr(const sht_plan* p, int kind) {
  switch (kind) {
    case kBasis: return p->basis;
    case kDBasis: return p->dbasis;
    case kAnalysis: return p->analysis;
    case kRot: return p->rot;
    default: return p->shear;
  }
}
int table_flip(int kind) { return (kind == kDBasis || kind == kShear) ? 1 : 0; }
int table_dir(int kind) { return (kind == kBasis || kind == kDBasis) ? 0 : 1; }

void check_plan(const sht_plan* p) {
  SHT_REQUIRE(p != nullptr, "plan is NULL");
  SHT_REQUIRE(p->geometry_only || p->basis != nullptr, "plan was not built");
}

void check_transform_plan(const sht_plan* p) {
  check_plan(p);
  SHT_REQUIRE(!p->geometry_only, "geometry-only plan cannot transform");
}

void check_ptr(const void* ptr, const char* name) {
  if (ptr == nullptr) throw Error{SHT_ERR_ARG, std::string(name) + " is NULL"};
}

void ensure_scratch(sht_plan* p, int64_t R) {
  if (R <= p->scratch_rows) return;
  SHT_CUDA_OR_THROW(cudaDeviceSynchronize());  // nothing may still read the old buffers
  for (int i = 0; i < 2; ++i) {
    if (p->wfold[i]) cudaFree(p->wfold[i]);
    if (p->cfold[i]) cudaFree(p->cfold[i]);
    p->wfold[i] = p->cfold[i] = nullptr;
  }
  if (p->rowmax) cudaFree(p->rowmax);
  p->rowmax = nullptr;
  p->scratch_rows = 0;
  for (int i = 0; i < 2; ++i) {
    SHT_CUDA_OR_THROW(cudaMalloc(&p->wfold[i], p->elem() * std::max<int64_t>(p->wfold_elems(R), 1)));
    SHT_CUDA_OR_THROW(cudaMalloc(&p->cfold[i], p->elem() * std::max<int64_t>(p->cfold_elems(R), 1)));
  }
  SHT_CUDA_OR_THROW(cudaMalloc(&p->rowmax, sizeof(float) * std::max<int64_t>(R, 1)));
  p->scratch_rows = R;
}

bool uses_tc(const sht_plan* p) {
  return p->prec == SHT_PREC_SPLIT16 && p->tc != nullptr && p->tune_contraction == 0;
}

// The row-max buffer the producer of a split-precision operand fills
// (zeroed first), or nullptr on the FP32/FP64 paths.
float* rowmax_for(sht_plan* p, int64_t R, cudaStream_t s) {
  if (!uses_tc(p)) return nullptr;
  SHT_CUDA_OR_THROW(cudaMemsetAsync(p->rowmax, 0, sizeof(float) * R, s));
  return p->rowmax;
}

template <typename T>
void contract(sht_plan* p, int kind, const T* data, T* out, int64_t R, cudaStream_t s) {
  const int dir = table_dir(kind), flip = table_flip(kind);
  KernelScope scope(p, dir == 0 ? SHT_KIND_LEGENDRE_SYNTHESIS : SHT_KIND_LEGENDRE_ANALYSIS, s);
  if constexpr (sizeof(T) == 4) {
    if (uses_tc(p)) {
      launch_gemm_tc(p, dir, flip, kind, data, p->rowmax, out, R, s);
      return;
    }
  }
  launch_gemm_simt<T>(p, dir, flip, static_cast<const T*>(table_ptr(p, kind)), data, out, R, s);
}

// Two contractions of the same data (P and dP/dphi tables of a gradient or
// wind synthesis; rotational and shear tables of a vordiv analysis): one
// tensor-core launch over the merged tiles on the split path.
template <typename T>
void contract2(sht_plan* p, int kind0, T* out0, int kind1, T* out1, const T* data, int64_t R,
               cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    if (uses_tc(p)) {
      const int dir = table_dir(kind0);
      KernelScope scope(p, dir == 0 ? SHT_KIND_LEGENDRE_SYNTHESIS : SHT_KIND_LEGENDRE_ANALYSIS, s);
      TcGroupSpec g[2] = {
          {p, dir, table_flip(kind0), kind0, data, p->rowmax, out0, R},
          {p, table_dir(kind1), table_flip(kind1), kind1, data, p->rowmax, out1, R}};
      launch_gemm_tc_groups(g, 2, tc_plan_cache(p), s);
      return;
    }
  }
  contract<T>(p, kind0, data, out0, R, s);
  contract<T>(p, kind1, data, out1, R, s);
}

// Two contractions of different operands, each with its own row maxima (the
// rotational table on the u rows and the shear table on the v rows of a
// divergence-only analysis): one tensor-core launch with two groups on the
// split path.
template <typename T>
void contract_pair(sht_plan* p, int kind0, const T* data0, const float* rm0, T* out0, int kind1,
                   const T* data1, const float* rm1, T* out1, int64_t R, cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    if (uses_tc(p)) {
      const int dir = table_dir(kind0);
      KernelScope scope(p, dir == 0 ? SHT_KIND_LEGENDRE_SYNTHESIS : SHT_KIND_LEGENDRE_ANALYSIS, s);
      TcGroupSpec g[2] = {{p, dir, table_flip(kind0), kind0, data0, rm0, out0, R},
                          {p, table_dir(kind1), table_flip(kind1), kind1, data1, rm1, out1, R}};
      launch_gemm_tc_groups(g, 2, tc_plan_cache(p), s);
      return;
    }
  }
  contract<T>(p, kind0, data0, out0, R, s);
  contract<T>(p, kind1, data1, out1, R, s);
}

template <typename T>
void do_forward(sht_plan* p, const T* grid, int64_t planes, T* coeff, cudaStream_t s) {
  const int64_t R = 2 * planes;
  ensure_scratch(p, R);
  T* w = static_cast<T*>(p->wfold[0]);
  T* c = static_cast<T*>(p->cfold[0]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_FFT_FORWARD, s);
    launch_forward_fold<T>(p, grid, nullptr, planes, w, s, rm);
  }
  contract<T>(p, kAnalysis, w, c, R, s);
  {
    KernelScope k(p, SHT_KIND_UNPACK, s);
    launch_unpack<T>(p, kUnpackScalar, c, nullptr, planes, coeff, nullptr, s);
  }
}

template <typename T>
void do_synthesis(sht_plan* p, int kind, int mode, const T* coeff, int64_t planes, T* grid,
                  cudaStream_t s) {
  const int64_t R = 2 * planes;
  ensure_scratch(p, R);
  T* w = static_cast<T*>(p->wfold[0]);
  T* c = static_cast<T*>(p->cfold[0]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_PACK, s);
    launch_pack<T>(p, coeff, nullptr, planes, kPackPlain, c, s, rm);
  }
  contract<T>(p, kind, c, w, R, s);
  {
    KernelScope k(p, SHT_KIND_FFT_INVERSE, s);
    launch_inverse_unfold<T>(p, mode, w, nullptr, planes, grid, nullptr, s);
  }
}

template <typename T>
void do_gradient(sht_plan* p, const T* coeff, int64_t planes, T* east, T* north,
                 cudaStream_t s) {
  const int64_t R = 2 * planes;
  ensure_scratch(p, R);
  T* c = static_cast<T*>(p->cfold[0]);
  T* w0 = static_cast<T*>(p->wfold[0]);
  T* w1 = static_cast<T*>(p->wfold[1]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_PACK, s);
    launch_pack<T>(p, coeff, nullptr, planes, kPackPlain, c, s, rm);
  }
  contract2<T>(p, kBasis, w0, kDBasis, w1, c, R, s);
  {
    KernelScope k(p, SHT_KIND_FFT_INVERSE, s);
    launch_inverse_unfold<T>(p, kUnfoldGradient, w0, w1, planes, east, north, s);
  }
}

template <typename T>
void do_wind(sht_plan* p, const T* vort, const T* div, int64_t planes, T* u, T* v,
             cudaStream_t s) {
  const int64_t R = 4 * planes;
  ensure_scratch(p, R);
  T* c = static_cast<T*>(p->cfold[0]);
  T* w0 = static_cast<T*>(p->wfold[0]);
  T* w1 = static_cast<T*>(p->wfold[1]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_PACK, s);
    launch_pack<T>(p, vort, div, planes, kPackInvLap, c, s, rm);
  }
  contract2<T>(p, kBasis, w0, kDBasis, w1, c, R, s);
  {
    KernelScope k(p, SHT_KIND_FFT_INVERSE, s);
    launch_inverse_unfold<T>(p, kUnfoldWind, w0, w1, planes, u, v, s);
  }
}

template <typename T>
void do_vordiv(sht_plan* p, const T* u, const T* v, int64_t planes, T* vort, T* div,
               cudaStream_t s) {
  const int64_t R = 4 * planes;
  ensure_scratch(p, R);
  T* w = static_cast<T*>(p->wfold[0]);
  T* c0 = static_cast<T*>(p->cfold[0]);
  T* c1 = static_cast<T*>(p->cfold[1]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_FFT_FORWARD, s);
    launch_forward_fold<T>(p, u, v, planes, w, s, rm);
  }
  contract2<T>(p, kRot, c0, kShear, c1, w, R, s);
  {
    KernelScope k(p, SHT_KIND_UNPACK, s);
    launch_unpack<T>(p, kUnpackVorDiv, c0, c1, planes, vort, div, s);
  }
}

// Vorticity and divergence from the reference-layout Fourier waist of a
// stacked (u, v) pair, (2, planes, nlat, T+1): the contraction half of
// vordiv_from_wind (vector.py:113-134).  The import interleaves the two
// fields per plane, the layout the rotational/shear contractions and the
// vordiv epilogue of do_vordiv read.
template <typename T>
void do_vordiv_waist(sht_plan* p, const T* waist, int64_t planes, T* vort, T* div,
                     cudaStream_t s) {
  const int64_t R = 4 * planes;
  ensure_scratch(p, R);
  T* w = static_cast<T*>(p->wfold[0]);
  T* c0 = static_cast<T*>(p->cfold[0]);
  T* c1 = static_cast<T*>(p->cfold[1]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_PACK, s);
    launch_waist_import<T>(p, waist, 2 * planes, 1.0, w, rm, s, 2);
  }
  contract2<T>(p, kRot, c0, kShear, c1, w, R, s);
  {
    KernelScope k(p, SHT_KIND_UNPACK, s);
    launch_unpack<T>(p, kUnpackVorDiv, c0, c1, planes, vort, div, s);
  }
}

// Divergence alone from the same stacked waist (divergence_from_fourier,
// vector.py:136-166): the rotational table on the u half and the shear table
// on the v half only, each contraction at half the rows of the full pair.
template <typename T>
void do_divergence_waist(sht_plan* p, const T* waist, int64_t planes, T* div, cudaStream_t s) {
  const int64_t R = 2 * planes;
  ensure_scratch(p, 2 * R);
  T* wu = static_cast<T*>(p->wfold[0]);
  T* wv = static_cast<T*>(p->wfold[1]);
  T* c0 = static_cast<T*>(p->cfold[0]);
  T* c1 = static_cast<T*>(p->cfold[1]);
  const int64_t per_field = (int64_t)p->nlat * (p->T + 1) * planes;  // complex values
  {
    float* rm = rowmax_for(p, 2 * R, s);
    KernelScope k(p, SHT_KIND_PACK, s);
    launch_waist_import<T>(p, waist, planes, 1.0, wu, rm, s);
    launch_waist_import<T>(p, waist + 2 * per_field, planes, 1.0, wv, rm ? rm + R : nullptr, s);
  }
  const float* rm = uses_tc(p) ? p->rowmax : nullptr;
  contract_pair<T>(p, kRot, wu, rm, c0, kShear, wv, rm ? rm + R : nullptr, c1, R, s);
  {
    KernelScope k(p, SHT_KIND_UNPACK, s);
    launch_unpack<T>(p, kUnpackDiv, c0, c1, planes, div, nullptr, s);
  }
}

// The stage solve with the divergence synthesis fused onto it: the kernel
// writes D' into the plan's folded synthesis operand (and its row maxima),
// then the Legendre synthesis and the inverse FFT of D' follow.
template <typename T>
void do_helmholtz_synthesis(sht_plan* p, const sht_vertical* op, double tau_w, const T* div,
                            const T* theta, const T* lnps, T* odiv, T* otheta, T* olnps,
                            T* grid, cudaStream_t s) {
  const int64_t planes = op->nlev, R = 2 * planes;
  ensure_scratch(p, R);
  T* c = static_cast<T*>(p->cfold[0]);
  T* w = static_cast<T*>(p->wfold[0]);
  {
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_HELMHOLTZ, s);
    launch_semi_implicit<T>(p, op->nlev, static_cast<const T*>(op->mats), op->thermo, kSemiSolve,
                            tau_w, 1.0, div, theta, lnps, odiv, otheta, olnps, nullptr, c, rm, s);
  }
  contract<T>(p, kBasis, c, w, R, s);
  {
    KernelScope k(p, SHT_KIND_FFT_INVERSE, s);
    launch_inverse_unfold<T>(p, kUnfoldScalar, w, nullptr, planes, grid, nullptr, s);
  }
}

// ------------------------------------------------------------------ batches
// A batch of plans (different truncations, or the same truncation under
// separate plans) run as one transform: per-plan FFT, pack and unpack
// launches around ONE Legendre launch per direction.  On the split path that
// launch is the persistent tensor-core kernel over the merged, cost-sorted
// tiles of every plan, so the large low-order tiles of the biggest
// truncation start first and the small tiles of all plans fill the tail.
template <typename T>
void contract_batch(sht_batch* b, int kind, T* const* data, T* const* out, cudaStream_t s) {
  const int n = (int)b->plans.size();
  if constexpr (sizeof(T) == 4) {
    bool all_tc = true;
    for (sht_plan* p : b->plans) all_tc = all_tc && uses_tc(p);
    if (all_tc) {
      const int dir = table_dir(kind);
      KernelScope scope(b->plans[0],
                        dir == 0 ? SHT_KIND_LEGENDRE_SYNTHESIS : SHT_KIND_LEGENDRE_ANALYSIS, s);
      TcGroupSpec g[kMaxTcGroups];
      for (int i = 0; i < n; ++i)
        g[i] = {b->plans[i], dir, table_flip(kind), kind, data[i], b->plans[i]->rowmax, out[i],
                2 * b->planes[i]};
      launch_gemm_tc_groups(g, n, b->cache, s);
      return;
    }
  }
  for (int i = 0; i < n; ++i) contract<T>(b->plans[i], kind, data[i], out[i], 2 * b->planes[i], s);
}

template <typename T>
void do_batch_forward(sht_batch* b, const void* const* grids, void* const* coeffs, cudaStream_t s) {
  const int n = (int)b->plans.size();
  T* w[kMaxTcGroups];
  T* c[kMaxTcGroups];
  for (int i = 0; i < n; ++i) {
    sht_plan* p = b->plans[i];
    const int64_t planes = b->planes[i], R = 2 * planes;
    ensure_scratch(p, R);
    w[i] = static_cast<T*>(p->wfold[0]);
    c[i] = static_cast<T*>(p->cfold[0]);
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_FFT_FORWARD, s);
    launch_forward_fold<T>(p, static_cast<const T*>(grids[i]), nullptr, planes, w[i], s, rm);
  }
  contract_batch<T>(b, kAnalysis, w, c, s);
  for (int i = 0; i < n; ++i) {
    KernelScope k(b->plans[i], SHT_KIND_UNPACK, s);
    launch_unpack<T>(b->plans[i], kUnpackScalar, c[i], nullptr, b->planes[i],
                     static_cast<T*>(coeffs[i]), nullptr, s);
  }
}

template <typename T>
void do_batch_inverse(sht_batch* b, const void* const* coeffs, void* const* grids, cudaStream_t s) {
  const int n = (int)b->plans.size();
  T* w[kMaxTcGroups];
  T* c[kMaxTcGroups];
  for (int i = 0; i < n; ++i) {
    sht_plan* p = b->plans[i];
    const int64_t planes = b->planes[i], R = 2 * planes;
    ensure_scratch(p, R);
    w[i] = static_cast<T*>(p->wfold[0]);
    c[i] = static_cast<T*>(p->cfold[0]);
    float* rm = rowmax_for(p, R, s);
    KernelScope k(p, SHT_KIND_PACK, s);
    launch_pack<T>(p, static_cast<const T*>(coeffs[i]), nullptr, planes, kPackPlain, c[i], s, rm);
  }
  contract_batch<T>(b, kBasis, c, w, s);
  for (int i = 0; i < n; ++i) {
    KernelScope k(b->plans[i], SHT_KIND_FFT_INVERSE, s);
    launch_inverse_unfold<T>(b->plans[i], kUnfoldScalar, w[i], nullptr, b->planes[i],
                             static_cast<T*>(grids[i]), nullptr, s);
  }
}

// ------------------------------------------------------- vertical operators
// Packs B, C, V, V^-1, lambda and (when w is given) W, W^-1, mu in the
// plan's type, in the order the semi-implicit kernel reads them.
sht_vertical* vertical_upload(const sht_plan* plan, int nlev, const double* b, const double* c,
                              const double* eigvec, const double* eigvec_inv,
                              const double* eigenvalues, const double* w = nullptr,
                              const double* w_inv = nullptr, const double* x_eigenvalues = nullptr) {
  SHT_REQUIRE(nlev >= 1 && nlev <= 96, "nlev must be in [1, 96]");
  for (const void* q : {(const void*)b, (const void*)c, (const void*)eigvec,
                        (const void*)eigvec_inv, (const void*)eigenvalues})
    check_ptr(q, "vertical operator matrix");
  const bool thermo = w != nullptr;
  if (thermo) {
    check_ptr(w_inv, "thermodynamic modes' inverse");
    check_ptr(x_eigenvalues, "thermodynamic eigenvalues");
  }
  const int L1 = nlev + 1;
  const size_t nm = (size_t)nlev * L1 * 2 + (size_t)nlev * nlev * 2 + nlev +
                    (thermo ? (size_t)L1 * L1 * 2 + L1 : 0);
  std::vector<double> host(nm);
  size_t o = 0;
  auto put = [&](const double* src, size_t n) {
    std::copy(src, src + n, host.begin() + o);
    o += n;
  };
  put(b, (size_t)nlev * L1);
  put(c, (size_t)L1 * nlev);
  put(eigvec, (size_t)nlev * nlev);
  put(eigvec_inv, (size_t)nlev * nlev);
  put(eigenvalues, nlev);
  if (thermo) {
    put(w, (size_t)L1 * L1);
    put(w_inv, (size_t)L1 * L1);
    put(x_eigenvalues, L1);
  }
  auto* op = new sht_vertical;
  op->device = plan->device;
  op->prec = plan->prec;
  op->nlev = nlev;
  op->thermo = thermo;
  try {
    if (plan->prec == SHT_PREC_F64) {
      SHT_CUDA_OR_THROW(cudaMalloc(&op->mats, sizeof(double) * nm));
      upload_now(op->mats, host.data(), sizeof(double) * nm);
    } else {
      std::vector<float> conv(host.begin(), host.end());
      SHT_CUDA_OR_THROW(cudaMalloc(&op->mats, sizeof(float) * nm));
      upload_now(op->mats, conv.data(), sizeof(float) * nm);
    }
    SHT_CUDA_OR_THROW(cudaMalloc(&op->metric, sizeof(double)));
  } catch (...) {
    if (op->mats) cudaFree(op->mats);
    if (op->metric) cudaFree(op->metric);
    delete op;
    throw;
  }
  return op;
}

void vertical_free(sht_vertical* op) {
  if (!op) return;
  if (op->mats) cudaFree(op->mats);
  if (op->metric) cudaFree(op->metric);
  delete op;
}

void host_stream_free(sht_plan* p) {
  auto& h = p->hs;
  for (int i = 0; i < sht_plan::kHostSlots; ++i) {
    for (int j = 0; j < 3; ++j)
      if (h.buf[i][j]) cudaFree(h.buf[i][j]);
    for (cudaEvent_t e : {h.h2d[i], h.comp[i], h.d2h[i]})
      if (e) cudaEventDestroy(e);
  }
  for (cudaStream_t st : {h.s_in, h.s_comp, h.s_out})
    if (st) cudaStreamDestroy(st);
  h = sht_plan::HostStream{};
}

void destroy(sht_plan* p) {
  if (!p) return;
  host_stream_free(p);
  destroy_tc_tables(p);
  for (auto& r : p->timing_recs) {
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
  }
  for (cudaEvent_t e : p->event_pool) cudaEventDestroy(e);
  void* ptrs[] = {p->d_mu, p->d_w, p->d_coslat, p->basis, p->dbasis, p->analysis, p->rot,
                  p->shear, p->tw_l, p->tw_n, p->d_radices, p->d_items[0], p->d_items[1],
                  p->d_items_narrow[0], p->d_items_narrow[1],
                  p->d_desc[0][0], p->d_desc[0][1], p->d_desc[1][0], p->d_desc[1][1],
                  p->wfold[0], p->wfold[1], p->cfold[0], p->cfold[1], p->rowmax, p->d_err};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete p;
}

// The streams, events and slot buffers of the host-streamed calls, grown to
// hold chunks of the given byte sizes.
void host_stream_prepare(sht_plan* p, const size_t (&bytes)[3]) {
  auto& h = p->hs;
  if (h.s_in == nullptr) {
    for (cudaStream_t* st : {&h.s_in, &h.s_comp, &h.s_out})
      SHT_CUDA_OR_THROW(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking));
    for (int i = 0; i < sht_plan::kHostSlots; ++i)
      for (cudaEvent_t* e : {&h.h2d[i], &h.comp[i], &h.d2h[i]})
        SHT_CUDA_OR_THROW(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  for (int j = 0; j < 3; ++j) {
    if (bytes[j] <= h.cap[j]) continue;
    SHT_CUDA_OR_THROW(cudaDeviceSynchronize());  // nothing may still use the old buffers
    for (int i = 0; i < sht_plan::kHostSlots; ++i) {
      if (h.buf[i][j]) cudaFree(h.buf[i][j]);
      h.buf[i][j] = nullptr;
    }
    h.cap[j] = 0;
    for (int i = 0; i < sht_plan::kHostSlots; ++i)
      SHT_CUDA_OR_THROW(cudaMalloc(&h.buf[i][j], bytes[j]));
    h.cap[j] = bytes[j];
  }
}

enum HostOp { kHostForward = 0, kHostInverse = 1, kHostRoundTrip = 2 };

// Plane counts of the chunks of a host-streamed call, each <= chunk.
// Uniform: chunk planes each, the remainder last.  Ramped (the default
// schedule): 2, 4, 8, ... planes below `chunk` at both ends and near-equal
// even chunks of at most `chunk` planes between, so the first copy-out
// starts after a short copy-in and the last copy-out after the end of the
// copy-in is short; the pipeline's fill and drain then cost a few planes'
// copies instead of two whole chunks'.
std::vector<int64_t> chunk_schedule(int64_t planes, int64_t chunk, bool ramped) {
  std::vector<int64_t> ramp;
  if (ramped) {
    int64_t sum = 0;
    for (int64_t c = 2; c < chunk; c *= 2) {
      ramp.push_back(c);
      sum += c;
    }
    if (planes < 2 * sum + 2 * chunk) ramp.clear();  // too short a batch to ramp
  }
  std::vector<int64_t> sizes(ramp);
  int64_t middle = planes;
  for (int64_t c : ramp) middle -= 2 * c;
  if (!ramped) {
    for (int64_t p0 = 0; p0 < middle; p0 += chunk) sizes.push_back(std::min(chunk, middle - p0));
  } else {
    // near-equal chunks in units of two planes; an odd plane goes last
    const int64_t pairs = middle / 2, n_mid = std::max<int64_t>(1, div_up(middle, chunk));
    for (int64_t i = 0; i < n_mid; ++i)
      sizes.push_back(2 * (pairs / n_mid + (i < pairs % n_mid ? 1 : 0)));
    sizes.back() += middle % 2;
  }
  for (auto it = ramp.rbegin(); it != ramp.rend(); ++it) sizes.push_back(*it);
  return sizes;
}

// Host in, host out, in chunks of `chunk` planes: chunk k's copy in (stream
// s_in), transforms (s_comp) and copy out (s_out) run in slot k % 3, so the
// copies of neighbouring chunks overlap each other and the transforms.  A
// slot's input is refilled once its transforms are done, its output once
// its copy-out is done.  Returns when the output is on the host.
template <typename T>
void host_streamed(sht_plan* p, int op, const void* hin, int64_t planes, void* hout,
                   int64_t chunk) {
  const int64_t ge = (int64_t)p->nlat * p->nlon;         // grid reals per plane
  const int64_t ce = (int64_t)(p->T + 1) * (p->T + 1) * 2;  // coefficient reals per plane
  const int64_t in_e = op == kHostInverse ? ce : ge, out_e = op == kHostForward ? ce : ge;
  const size_t es = sizeof(T);
  // Default: about a sixteenth of the planes, even (the register FFTs' pair
  // kernel wants even plane counts); at T511 x 200 planes chunks of 8-26
  // planes time alike, within 2 %, and whole-batch copies 60 % slower.
  const bool ramped = chunk <= 0;
  if (chunk <= 0) chunk = std::max<int64_t>(2, (div_up(planes, 16) + 1) / 2 * 2);
  chunk = std::min(chunk, planes);
  const std::vector<int64_t> sizes = chunk_schedule(planes, chunk, ramped);
  {
    int64_t sum = 0;
    for (int64_t n : sizes) {
      SHT_REQUIRE(n >= 1 && n <= chunk, "internal: a chunk outside [1, chunk] planes");
      sum += n;
    }
    SHT_REQUIRE(sum == planes, "internal: the chunks do not cover the planes");
  }
  const size_t bytes[3] = {(size_t)(chunk * in_e) * es,
                           op == kHostRoundTrip ? (size_t)(chunk * ce) * es : 0,
                           (size_t)(chunk * out_e) * es};
  host_stream_prepare(p, bytes);
  ensure_scratch(p, 2 * chunk);
  auto& h = p->hs;
  p->last_stream = h.s_comp;
  try {
    const int64_t n_chunks = (int64_t)sizes.size();
    int64_t p0 = 0;
    for (int64_t k = 0; k < n_chunks; p0 += sizes[k], ++k) {
      const int sl = (int)(k % sht_plan::kHostSlots);
      const int64_t n = sizes[k];
      if (k >= sht_plan::kHostSlots) SHT_CUDA_OR_THROW(cudaStreamWaitEvent(h.s_in, h.comp[sl], 0));
      SHT_CUDA_OR_THROW(cudaMemcpyAsync(h.buf[sl][0], static_cast<const char*>(hin) + p0 * in_e * es,
                                        (size_t)(n * in_e) * es, cudaMemcpyHostToDevice, h.s_in));
      SHT_CUDA_OR_THROW(cudaEventRecord(h.h2d[sl], h.s_in));
      SHT_CUDA_OR_THROW(cudaStreamWaitEvent(h.s_comp, h.h2d[sl], 0));
      if (k >= sht_plan::kHostSlots) SHT_CUDA_OR_THROW(cudaStreamWaitEvent(h.s_comp, h.d2h[sl], 0));
      const T* in = static_cast<const T*>(h.buf[sl][0]);
      T* mid = static_cast<T*>(h.buf[sl][1]);
      T* out = static_cast<T*>(h.buf[sl][2]);
      if (op == kHostForward) {
        do_forward<T>(p, in, n, out, h.s_comp);
      } else if (op == kHostInverse) {
        do_synthesis<T>(p, kBasis, kUnfoldScalar, in, n, out, h.s_comp);
      } else {
        do_forward<T>(p, in, n, mid, h.s_comp);
        do_synthesis<T>(p, kBasis, kUnfoldScalar, mid, n, out, h.s_comp);
      }
      SHT_CUDA_OR_THROW(cudaEventRecord(h.comp[sl], h.s_comp));
      SHT_CUDA_OR_THROW(cudaStreamWaitEvent(h.s_out, h.comp[sl], 0));
      SHT_CUDA_OR_THROW(cudaMemcpyAsync(static_cast<char*>(hout) + p0 * out_e * es, out,
                                        (size_t)(n * out_e) * es, cudaMemcpyDeviceToHost, h.s_out));
      SHT_CUDA_OR_THROW(cudaEventRecord(h.d2h[sl], h.s_out));
    }
  } catch (...) {
    // Leave nothing in flight on the caller's buffers.
    for (cudaStream_t st : {h.s_in, h.s_comp, h.s_out}) cudaStreamSynchronize(st);
    throw;
  }
  for (cudaStream_t st : {h.s_in, h.s_comp, h.s_out})
    SHT_CUDA_OR_THROW(cudaStreamSynchronize(st));
}

#define DISPATCH(p, FN, ...)                       \
  do {                                             \
    if ((p)->prec == SHT_PREC_F64)                 \
      FN<double>(__VA_ARGS__);                     \
    else                                           \
      FN<float>(__VA_ARGS__);                      \
  } while (0)

}  // namespace
}  // namespace sht

using namespace sht;

namespace {

// The folded table of one kind: device pointer, and whether it is held in the
// synthesis layout [m][q][i][h] (ld Hx) or the analysis layout [m][q][h][i]
// (ld ex).
const void* folded_table(const sht_plan* p, int table, bool* synthesis_layout) {
  SHT_REQUIRE(table >= SHT_TABLE_BASIS && table <= SHT_TABLE_SHEAR,
              "table must be one of SHT_TABLE_BASIS .. SHT_TABLE_SHEAR");
  SHT_REQUIRE(!p->geometry_only, "a geometry-only plan holds no Legendre tables");
  const void* t[5] = {p->basis, p->dbasis, p->analysis, p->rot, p->shear};
  *synthesis_layout = table <= SHT_TABLE_DBASIS;
  return t[table];
}

// Dense expansion of a folded table (host copy `f`) into `out`.  Row j < H is
// the folded row h = j; row j >= H mirrors h = nlat - 1 - j with the sign
// (-1)^(n-m) of P_nm under mu -> -mu, negated for the tables built from
// dP/dphi.
template <typename T>
void expand_dense(const sht_plan* p, int table, bool syn, const T* f, T* out) {
  const int T1 = p->T + 1, nlat = p->nlat, H = p->H;
  const bool odd_in_lat = table == SHT_TABLE_DBASIS || table == SHT_TABLE_SHEAR;
  std::fill(out, out + (int64_t)T1 * T1 * nlat, T(0));
  for (int m = 0; m < T1; ++m)
    for (int n = m; n < T1; ++n) {
      const int q = (n - m) & 1, i = (n - m) >> 1, idx = m * 2 + q;
      const bool flip = (q == 1) != odd_in_lat;
      for (int j = 0; j < nlat; ++j) {
        const bool north = j >= H;
        const int h = north ? nlat - 1 - j : j;
        T v = syn ? f[p->syn_off[idx] + (int64_t)i * p->Hx + h]
                  : f[p->ana_off[idx] + (int64_t)h * p->ex[idx] + i];
        if (north && flip) v = -v;
        if (syn)
          out[((int64_t)m * T1 + n) * nlat + j] = v;
        else
          out[((int64_t)m * nlat + j) * T1 + n] = v;
      }
    }
}

}  // namespace

extern "C" {

int sht_abi_version(void) { return SHT_ABI_VERSION; }

const char* sht_last_error(void) { return g_error.c_str(); }

int sht_plan_create(int truncation, int nlat, int nlon, double radius_m, int precision,
                    int flags, sht_plan** out_plan) {
  return guarded([&] {
    SHT_REQUIRE(out_plan != nullptr, "out_plan is NULL");
    *out_plan = nullptr;
    SHT_REQUIRE(truncation >= 1, "truncation must be >= 1");
    SHT_REQUIRE(nlat >= truncation + 1, "nlat must be >= truncation + 1");
    SHT_REQUIRE(nlon % 2 == 0, "nlon must be even");
    SHT_REQUIRE(nlon >= 2 * truncation + 2, "nlon must be >= 2 * truncation + 2");
    SHT_REQUIRE(radius_m > 0, "radius_m must be positive");
    SHT_REQUIRE(precision == SHT_PREC_F64 || precision == SHT_PREC_F32 ||
                    precision == SHT_PREC_SPLIT16,
                "precision must be SHT_PREC_F64, SHT_PREC_F32 or SHT_PREC_SPLIT16");
    SHT_REQUIRE((flags & ~(SHT_FLAG_GEOMETRY_ONLY | SHT_FLAG_GENERIC_FFT)) == 0,
                "flags must be a combination of SHT_FLAG_GEOMETRY_ONLY and SHT_FLAG_GENERIC_FFT");
    sht_plan* p = new sht_plan();
    p->T = truncation;
    p->nlat = nlat;
    p->nlon = nlon;
    p->radius = radius_m;
    p->prec = precision;
    cudaStream_t s = nullptr;
    try {
      SHT_CUDA_OR_THROW(cudaGetDevice(&p->device));
      SHT_CUDA_OR_THROW(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      SHT_CUDA_OR_THROW(cudaMalloc(&p->d_err, sizeof(unsigned) * 4));
      SHT_CUDA_OR_THROW(cudaMemsetAsync(p->d_err, 0, sizeof(unsigned) * 4, s));
      p->geometry_only = (flags & SHT_FLAG_GEOMETRY_ONLY) != 0;
      p->force_generic_fft = (flags & SHT_FLAG_GENERIC_FFT) != 0;
      build_geometry_and_tables(p, s);
      if (!p->geometry_only) {
        build_fft(p, s);
        build_gemm_items(p);
      }
      SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
      SHT_CUDA_OR_THROW(cudaStreamDestroy(s));
    } catch (...) {
      if (s) cudaStreamDestroy(s);
      destroy(p);
      throw;
    }
    *out_plan = p;
  });
}

int sht_plan_destroy(sht_plan* plan) {
  return guarded([&] {
    if (plan) cudaDeviceSynchronize();
    destroy(plan);
  });
}

int sht_plan_reserve(sht_plan* plan, int64_t planes) {
  return guarded([&] {
    check_transform_plan(plan);
    SHT_REQUIRE(planes >= 0, "planes must be >= 0");
    ensure_scratch(plan, 4 * planes);
  });
}

int sht_plan_geometry(const sht_plan* plan, double* mu, double* weights, double* coslat) {
  return guarded([&] {
    check_plan(plan);
    size_t n = plan->nlat;
    if (mu) std::copy(plan->h_mu.begin(), plan->h_mu.begin() + n, mu);
    if (weights) std::copy(plan->h_w.begin(), plan->h_w.begin() + n, weights);
    if (coslat) std::copy(plan->h_coslat.begin(), plan->h_coslat.begin() + n, coslat);
  });
}

int sht_plan_table_bytes(const sht_plan* plan, int table, int64_t* bytes) {
  return guarded([&] {
    check_plan(plan);
    SHT_REQUIRE(bytes != nullptr, "bytes must not be NULL");
    bool syn = false;
    folded_table(plan, table, &syn);
    const int64_t elems = syn ? plan->syn_total : plan->ana_total;
    *bytes = elems * (int64_t)plan->elem() + sht::tc_table_bytes(plan, table);
  });
}

int sht_plan_read_table(const sht_plan* plan, int table, void* host_out) {
  return guarded([&] {
    check_plan(plan);
    SHT_REQUIRE(host_out != nullptr, "host_out must not be NULL");
    bool syn = false;
    const void* d = folded_table(plan, table, &syn);
    const int64_t elems = syn ? plan->syn_total : plan->ana_total;
    if (plan->prec == SHT_PREC_F64) {
      std::vector<double> f((size_t)std::max<int64_t>(elems, 1));
      SHT_CUDA_OR_THROW(cudaMemcpy(f.data(), d, 8 * elems, cudaMemcpyDeviceToHost));
      expand_dense(plan, table, syn, f.data(), static_cast<double*>(host_out));
    } else {
      std::vector<float> f((size_t)std::max<int64_t>(elems, 1));
      SHT_CUDA_OR_THROW(cudaMemcpy(f.data(), d, 4 * elems, cudaMemcpyDeviceToHost));
      expand_dense(plan, table, syn, f.data(), static_cast<float*>(host_out));
    }
  });
}

int sht_plan_set_timing(sht_plan* plan, int enable) {
  return guarded([&] {
    check_plan(plan);
    plan->timing = enable != 0;
  });
}

int sht_plan_read_timing(sht_plan* plan, double* ms, int64_t* launches, int64_t* timed, int n,
                         int reset) {
  return guarded([&] {
    check_plan(plan);
    SHT_REQUIRE(n >= 0 && n <= SHT_KIND_COUNT, "n must be in [0, SHT_KIND_COUNT]");
    for (auto& r : plan->timing_recs) {
      SHT_CUDA_OR_THROW(cudaEventSynchronize(r.stop));
      float e = 0.f;
      SHT_CUDA_OR_THROW(cudaEventElapsedTime(&e, r.start, r.stop));
      plan->ms[r.kind] += e;
      plan->timed[r.kind]++;
      plan->event_pool.push_back(r.start);
      plan->event_pool.push_back(r.stop);
    }
    plan->timing_recs.clear();
    for (int i = 0; i < n; ++i) {
      if (ms) ms[i] = plan->ms[i];
      if (launches) launches[i] = plan->launches[i];
      if (timed) timed[i] = plan->timed[i];
    }
    if (reset)
      for (int i = 0; i < SHT_KIND_COUNT; ++i) plan->ms[i] = 0, plan->launches[i] = 0, plan->timed[i] = 0;
  });
}

int sht_plan_check(sht_plan* plan) {
  return guarded([&] {
    check_plan(plan);
    SHT_CUDA_OR_THROW(cudaDeviceSynchronize());
    unsigned h[4] = {0, 0, 0, 0};
    SHT_CUDA_OR_THROW(cudaMemcpy(h, plan->d_err, sizeof(h), cudaMemcpyDeviceToHost));
    SHT_CUDA_OR_THROW(cudaMemset(plan->d_err, 0, sizeof(h)));
    if (h[0] != 0) {
      char buf[256];
      snprintf(buf, sizeof(buf),
               "device error word 0x%x: %s (tile %u, stage %u)", h[0],
               (h[0] & kErrBadTile) ? "a tensor-core launch met an invalid tile and stopped"
                                    : "a kernel gave up on a bounded wait",
               h[1], h[2]);
      throw Error{SHT_ERR_DEVICE, buf};
    }
  });
}

#define SHT_CHECK_CALL(plan, planes)                                   \
  check_transform_plan(plan);                                          \
  SHT_REQUIRE((planes) >= 0, "planes must be >= 0");                   \
  if ((planes) == 0) return;                                           \
  cudaStream_t s = static_cast<cudaStream_t>(stream);                  \
  plan->last_stream = s

#define SHT_TYPED(plan, CALL)                                          \
  do {                                                                 \
    if ((plan)->prec == SHT_PREC_F64) {                                \
      using T = double;                                                \
      CALL;                                                            \
    } else {                                                           \
      using T = float;                                                 \
      CALL;                                                            \
    }                                                                  \
  } while (0)

#define CP(x) static_cast<const T*>(x)
#define MP(x) static_cast<T*>(x)

int sht_forward(sht_plan* plan, const void* grid, int64_t planes, void* coeff, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(grid, "grid");
    check_ptr(coeff, "coeff");
    SHT_TYPED(plan, do_forward<T>(plan, CP(grid), planes, MP(coeff), s));
  });
}

int sht_inverse(sht_plan* plan, const void* coeff, int64_t planes, void* grid, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(coeff, "coeff");
    check_ptr(grid, "grid");
    SHT_TYPED(plan, do_synthesis<T>(plan, kBasis, kUnfoldScalar, CP(coeff), planes, MP(grid), s));
  });
}

int sht_forward_host(sht_plan* plan, const void* host_grid, int64_t planes, void* host_coeff,
                     int64_t chunk) {
  return guarded([&] {
    void* stream = nullptr;
    SHT_CHECK_CALL(plan, planes);
    check_ptr(host_grid, "host_grid");
    check_ptr(host_coeff, "host_coeff");
    SHT_REQUIRE(chunk >= 0, "chunk must be >= 0");
    SHT_TYPED(plan, host_streamed<T>(plan, kHostForward, host_grid, planes, host_coeff, chunk));
  });
}

int sht_inverse_host(sht_plan* plan, const void* host_coeff, int64_t planes, void* host_grid,
                     int64_t chunk) {
  return guarded([&] {
    void* stream = nullptr;
    SHT_CHECK_CALL(plan, planes);
    check_ptr(host_coeff, "host_coeff");
    check_ptr(host_grid, "host_grid");
    SHT_REQUIRE(chunk >= 0, "chunk must be >= 0");
    SHT_TYPED(plan, host_streamed<T>(plan, kHostInverse, host_coeff, planes, host_grid, chunk));
  });
}

int sht_round_trip_host(sht_plan* plan, const void* host_grid, int64_t planes, void* host_out,
                        int64_t chunk) {
  return guarded([&] {
    void* stream = nullptr;
    SHT_CHECK_CALL(plan, planes);
    check_ptr(host_grid, "host_grid");
    check_ptr(host_out, "host_out");
    SHT_REQUIRE(chunk >= 0, "chunk must be >= 0");
    SHT_TYPED(plan, host_streamed<T>(plan, kHostRoundTrip, host_grid, planes, host_out, chunk));
  });
}

int sht_inverse_meridional_derivative(sht_plan* plan, const void* coeff, int64_t planes,
                                      void* grid, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(coeff, "coeff");
    check_ptr(grid, "grid");
    SHT_TYPED(plan, do_synthesis<T>(plan, kDBasis, kUnfoldMeridional, CP(coeff), planes,
                                    MP(grid), s));
  });
}

int sht_inverse_zonal_derivative(sht_plan* plan, const void* coeff, int64_t planes, void* grid,
                                 void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(coeff, "coeff");
    check_ptr(grid, "grid");
    SHT_TYPED(plan, do_synthesis<T>(plan, kBasis, kUnfoldZonal, CP(coeff), planes, MP(grid), s));
  });
}

int sht_gradient(sht_plan* plan, const void* coeff, int64_t planes, void* east, void* north,
                 void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(coeff, "coeff");
    check_ptr(east, "east");
    check_ptr(north, "north");
    SHT_TYPED(plan, do_gradient<T>(plan, CP(coeff), planes, MP(east), MP(north), s));
  });
}

int sht_wind_from_vordiv(sht_plan* plan, const void* vorticity, const void* divergence,
                         int64_t planes, void* u, void* v, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(vorticity, "vorticity");
    check_ptr(divergence, "divergence");
    check_ptr(u, "u");
    check_ptr(v, "v");
    SHT_TYPED(plan, do_wind<T>(plan, CP(vorticity), CP(divergence), planes, MP(u), MP(v), s));
  });
}

int sht_vordiv_from_wind(sht_plan* plan, const void* u, const void* v, int64_t planes,
                         void* vorticity, void* divergence, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(u, "u");
    check_ptr(v, "v");
    check_ptr(vorticity, "vorticity");
    check_ptr(divergence, "divergence");
    SHT_TYPED(plan, do_vordiv<T>(plan, CP(u), CP(v), planes, MP(vorticity), MP(divergence), s));
  });
}

int sht_vordiv_from_waist(sht_plan* plan, const void* waist, int64_t planes, void* vorticity,
                          void* divergence, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(waist, "waist");
    check_ptr(vorticity, "vorticity");
    check_ptr(divergence, "divergence");
    SHT_TYPED(plan, do_vordiv_waist<T>(plan, CP(waist), planes, MP(vorticity), MP(divergence), s));
  });
}

int sht_divergence_from_waist(sht_plan* plan, const void* waist, int64_t planes, void* divergence,
                              void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(waist, "waist");
    check_ptr(divergence, "divergence");
    SHT_TYPED(plan, do_divergence_waist<T>(plan, CP(waist), planes, MP(divergence), s));
  });
}

static int elementwise_entry(sht_plan* plan, int mode, const void* in, int64_t planes, void* out,
                             void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(in, "in");
    check_ptr(out, "out");
    KernelScope k(plan, SHT_KIND_ELEMENTWISE, s);
    SHT_TYPED(plan, launch_elementwise<T>(plan, mode, CP(in), planes, MP(out), s));
  });
}

int sht_project(sht_plan* plan, const void* in, int64_t planes, void* out, void* stream) {
  return elementwise_entry(plan, kElemProject, in, planes, out, stream);
}
int sht_laplacian(sht_plan* plan, const void* in, int64_t planes, void* out, void* stream) {
  return elementwise_entry(plan, kElemLaplacian, in, planes, out, stream);
}
int sht_inverse_laplacian(sht_plan* plan, const void* in, int64_t planes, void* out,
                          void* stream) {
  return elementwise_entry(plan, kElemInvLaplacian, in, planes, out, stream);
}

static void vertical_apply(sht_plan* plan, const sht_vertical* op, double tau_w,
                           const void* divergence, const void* theta, const void* lnps,
                           void* out_divergence, void* out_theta, void* out_lnps,
                           cudaStream_t s) {
  for (const void* q : {divergence, theta, lnps, (const void*)out_divergence,
                        (const void*)out_theta, (const void*)out_lnps})
    check_ptr(q, "helmholtz argument");
  plan->last_stream = s;
  KernelScope k(plan, SHT_KIND_HELMHOLTZ, s);
  SHT_TYPED(plan, launch_helmholtz<T>(plan, op->nlev, static_cast<const T*>(op->mats), tau_w,
                                      CP(divergence), CP(theta), CP(lnps), MP(out_divergence),
                                      MP(out_theta), MP(out_lnps), s));
}

static void check_vertical(const sht_plan* plan, const sht_vertical* op) {
  check_transform_plan(plan);
  check_ptr(op, "vertical operator");
  SHT_REQUIRE(op->device == plan->device && op->prec == plan->prec,
              "the vertical operator was created for another plan's device or precision");
}

int sht_semi_implicit_map(sht_plan* plan, const sht_vertical* op, int mode, double dt_w,
                          double alpha, const void* divergence, const void* theta,
                          const void* lnps, void* out_divergence, void* out_theta,
                          void* out_lnps, void* stream) {
  return guarded([&] {
    check_vertical(plan, op);
    for (const void* q : {divergence, theta, lnps, (const void*)out_divergence,
                          (const void*)out_theta, (const void*)out_lnps})
      check_ptr(q, "semi-implicit argument");
    SHT_REQUIRE(mode == SHT_SEMI_SOLVE_SHIFTED || mode == SHT_SEMI_APPLY ||
                    mode == SHT_SEMI_HALF_APPLY || mode == SHT_SEMI_LINEAR_TENDENCIES,
                "mode must be SHT_SEMI_SOLVE_SHIFTED, SHT_SEMI_APPLY, SHT_SEMI_HALF_APPLY or "
                "SHT_SEMI_LINEAR_TENDENCIES");
    const bool uses_alpha = mode == SHT_SEMI_APPLY || mode == SHT_SEMI_HALF_APPLY;
    SHT_REQUIRE(!uses_alpha || (alpha >= 0.5 && alpha <= 1.0),
                "off_centring_weight must lie in [0.5, 1]");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    plan->last_stream = s;
    const int kmode = mode == SHT_SEMI_APPLY ? kSemiApply
                      : mode == SHT_SEMI_HALF_APPLY ? kSemiHalf
                      : mode == SHT_SEMI_LINEAR_TENDENCIES ? kSemiLinear : kSemiSolve;
    SHT_CUDA_OR_THROW(cudaMemsetAsync(op->metric, 0, sizeof(double), s));
    KernelScope k(plan, SHT_KIND_HELMHOLTZ, s);
    SHT_TYPED(plan, launch_semi_implicit<T>(plan, op->nlev, static_cast<const T*>(op->mats),
                                            op->thermo, kmode, dt_w, uses_alpha ? alpha : 1.0,
                                            CP(divergence), CP(theta), CP(lnps),
                                            MP(out_divergence), MP(out_theta), MP(out_lnps),
                                            static_cast<T*>(op->metric), nullptr, nullptr, s));
  });
}

int sht_semi_implicit_metric(const sht_vertical* op, double* max_divergence_increment,
                             void* stream) {
  return guarded([&] {
    check_ptr(op, "vertical operator");
    check_ptr(max_divergence_increment, "max_divergence_increment");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double v = 0.0;
    if (op->prec == SHT_PREC_F64) {
      SHT_CUDA_OR_THROW(cudaMemcpyAsync(&v, op->metric, sizeof(double), cudaMemcpyDeviceToHost, s));
      SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
    } else {
      float f = 0.f;
      SHT_CUDA_OR_THROW(cudaMemcpyAsync(&f, op->metric, sizeof(float), cudaMemcpyDeviceToHost, s));
      SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
      v = f;
    }
    *max_divergence_increment = v;
  });
}

int sht_helmholtz_synthesis(sht_plan* plan, const sht_vertical* op, double tau_w,
                            const void* divergence, const void* theta, const void* lnps,
                            void* out_divergence, void* out_theta, void* out_lnps,
                            void* divergence_grid, void* stream) {
  return guarded([&] {
    check_vertical(plan, op);
    for (const void* q : {divergence, theta, lnps, (const void*)out_divergence,
                          (const void*)out_theta, (const void*)out_lnps,
                          (const void*)divergence_grid})
      check_ptr(q, "helmholtz_synthesis argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    plan->last_stream = s;
    SHT_TYPED(plan, do_helmholtz_synthesis<T>(plan, op, tau_w, CP(divergence), CP(theta),
                                              CP(lnps), MP(out_divergence), MP(out_theta),
                                              MP(out_lnps), MP(divergence_grid), s));
  });
}

int sht_helmholtz_solve(sht_plan* plan, int nlev, const double* b, const double* c,
                        const double* eigvec, const double* eigvec_inv,
                        const double* eigenvalues, double tau_w, const void* divergence,
                        const void* theta, const void* lnps, void* out_divergence,
                        void* out_theta, void* out_lnps, void* stream) {
  return guarded([&] {
    check_transform_plan(plan);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // One-shot form: upload, solve, and free once the solve has finished.
    sht_vertical* op = vertical_upload(plan, nlev, b, c, eigvec, eigvec_inv, eigenvalues);
    try {
      vertical_apply(plan, op, tau_w, divergence, theta, lnps, out_divergence, out_theta,
                     out_lnps, s);
      SHT_CUDA_OR_THROW(cudaStreamSynchronize(s));
    } catch (...) {
      vertical_free(op);
      throw;
    }
    vertical_free(op);
  });
}

int sht_vertical_create(sht_plan* plan, int nlev, const double* b, const double* c,
                        const double* eigvec, const double* eigvec_inv,
                        const double* eigenvalues, sht_vertical** out) {
  return guarded([&] {
    check_ptr(out, "out");
    *out = nullptr;
    check_transform_plan(plan);
    int device = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&device));
    SHT_REQUIRE(device == plan->device, "the current device is not the plan's device");
    *out = vertical_upload(plan, nlev, b, c, eigvec, eigvec_inv, eigenvalues);
  });
}

int sht_vertical_create_modes(sht_plan* plan, int nlev, const double* b, const double* c,
                              const double* eigvec, const double* eigvec_inv,
                              const double* eigenvalues, const double* x_eigvec,
                              const double* x_eigvec_inv, const double* x_eigenvalues,
                              sht_vertical** out) {
  return guarded([&] {
    check_ptr(out, "out");
    *out = nullptr;
    check_transform_plan(plan);
    check_ptr(x_eigvec, "x_eigvec");
    int device = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&device));
    SHT_REQUIRE(device == plan->device, "the current device is not the plan's device");
    *out = vertical_upload(plan, nlev, b, c, eigvec, eigvec_inv, eigenvalues, x_eigvec,
                           x_eigvec_inv, x_eigenvalues);
  });
}

int sht_vertical_destroy(sht_vertical* op) {
  return guarded([&] { vertical_free(op); });
}

int sht_helmholtz_apply(sht_plan* plan, const sht_vertical* op, double tau_w,
                        const void* divergence, const void* theta, const void* lnps,
                        void* out_divergence, void* out_theta, void* out_lnps, void* stream) {
  return guarded([&] {
    check_vertical(plan, op);
    vertical_apply(plan, op, tau_w, divergence, theta, lnps, out_divergence, out_theta, out_lnps,
                   static_cast<cudaStream_t>(stream));
  });
}

int sht_batch_create(int nplans, sht_plan* const* plans, const int64_t* planes,
                     sht_batch** out) {
  return guarded([&] {
    check_ptr(out, "out");
    *out = nullptr;
    SHT_REQUIRE(nplans >= 1 && nplans <= kMaxTcGroups, "a batch holds 1 to 4 plans");
    check_ptr(plans, "plans");
    check_ptr(planes, "planes");
    for (int i = 0; i < nplans; ++i) {
      check_transform_plan(plans[i]);
      SHT_REQUIRE(planes[i] >= 1, "every plan of a batch needs planes >= 1");
      SHT_REQUIRE(plans[i]->prec == plans[0]->prec, "the plans of a batch share one precision");
      SHT_REQUIRE(plans[i]->device == plans[0]->device, "the plans of a batch share one device");
      for (int j = 0; j < i; ++j)
        SHT_REQUIRE(plans[j] != plans[i],
                    "a plan appears twice in a batch (its scratch would be shared)");
    }
    auto* b = new sht_batch;
    b->plans.assign(plans, plans + nplans);
    b->planes.assign(planes, planes + nplans);
    b->cache = tc_cache_create();
    *out = b;
  });
}

int sht_batch_destroy(sht_batch* batch) {
  return guarded([&] {
    if (!batch) return;
    tc_cache_destroy(batch->cache);
    delete batch;
  });
}

static void check_batch_call(sht_batch* b, const void* const* in, void* const* out) {
  check_ptr(b, "batch");
  check_ptr(in, "input array list");
  check_ptr(out, "output array list");
  for (size_t i = 0; i < b->plans.size(); ++i) {
    check_transform_plan(b->plans[i]);
    check_ptr(in[i], "batch input");
    check_ptr(out[i], "batch output");
  }
}

int sht_batch_forward(sht_batch* batch, const void* const* grids, void* const* coeffs,
                      void* stream) {
  return guarded([&] {
    check_batch_call(batch, grids, coeffs);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (sht_plan* p : batch->plans) p->last_stream = s;
    if (batch->plans[0]->prec == SHT_PREC_F64)
      do_batch_forward<double>(batch, grids, coeffs, s);
    else
      do_batch_forward<float>(batch, grids, coeffs, s);
  });
}

int sht_batch_inverse(sht_batch* batch, const void* const* coeffs, void* const* grids,
                      void* stream) {
  return guarded([&] {
    check_batch_call(batch, coeffs, grids);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (sht_plan* p : batch->plans) p->last_stream = s;
    if (batch->plans[0]->prec == SHT_PREC_F64)
      do_batch_inverse<double>(batch, coeffs, grids, s);
    else
      do_batch_inverse<float>(batch, coeffs, grids, s);
  });
}

// ------------------------------------------------------------ Fourier waist
int sht_fourier_waist(sht_plan* plan, const void* grid, int64_t planes, void* waist,
                      void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(grid, "grid");
    check_ptr(waist, "waist");
    SHT_TYPED(plan, {
      ensure_scratch(plan, 2 * planes);
      T* w = static_cast<T*>(plan->wfold[0]);
      {
        KernelScope k(plan, SHT_KIND_FFT_FORWARD, s);
        launch_forward_fold<T>(plan, CP(grid), nullptr, planes, w, s, nullptr);
      }
      KernelScope k(plan, SHT_KIND_UNPACK, s);
      launch_waist_export<T>(plan, w, planes, 0.5, 0, MP(waist), s);
    });
  });
}

int sht_contract_waist(sht_plan* plan, const void* waist, int64_t planes, void* coeff,
                       void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(waist, "waist");
    check_ptr(coeff, "coeff");
    SHT_TYPED(plan, {
      const int64_t R = 2 * planes;
      ensure_scratch(plan, R);
      T* w = static_cast<T*>(plan->wfold[0]);
      T* c = static_cast<T*>(plan->cfold[0]);
      {
        float* rm = rowmax_for(plan, R, s);
        KernelScope k(plan, SHT_KIND_PACK, s);
        launch_waist_import<T>(plan, CP(waist), planes, 1.0, w, rm, s);
      }
      contract<T>(plan, kAnalysis, w, c, R, s);
      KernelScope k(plan, SHT_KIND_UNPACK, s);
      launch_unpack<T>(plan, kUnpackScalar, c, nullptr, planes, MP(coeff), nullptr, s);
    });
  });
}

int sht_contract_to_waist(sht_plan* plan, const void* coeff, int64_t planes, int table,
                          void* waist, void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(coeff, "coeff");
    check_ptr(waist, "waist");
    SHT_REQUIRE(table == SHT_WAIST_BASIS || table == SHT_WAIST_DBASIS || table == SHT_WAIST_ZONAL,
                "table must be SHT_WAIST_BASIS, SHT_WAIST_DBASIS or SHT_WAIST_ZONAL");
    SHT_TYPED(plan, {
      const int64_t R = 2 * planes;
      ensure_scratch(plan, R);
      T* w = static_cast<T*>(plan->wfold[0]);
      T* c = static_cast<T*>(plan->cfold[0]);
      {
        float* rm = rowmax_for(plan, R, s);
        KernelScope k(plan, SHT_KIND_PACK, s);
        launch_pack<T>(plan, CP(coeff), nullptr, planes, kPackPlain, c, s, rm);
      }
      contract<T>(plan, table == SHT_WAIST_DBASIS ? kDBasis : kBasis, c, w, R, s);
      KernelScope k(plan, SHT_KIND_UNPACK, s);
      launch_waist_export<T>(plan, w, planes, 1.0, table == SHT_WAIST_ZONAL ? 1 : 0, MP(waist), s);
    });
  });
}

int sht_waist_to_grid(sht_plan* plan, const void* waist, int64_t planes, void* grid,
                      void* stream) {
  return guarded([&] {
    SHT_CHECK_CALL(plan, planes);
    check_ptr(waist, "waist");
    check_ptr(grid, "grid");
    SHT_TYPED(plan, {
      ensure_scratch(plan, 2 * planes);
      T* w = static_cast<T*>(plan->wfold[0]);
      {
        KernelScope k(plan, SHT_KIND_PACK, s);
        launch_waist_import<T>(plan, CP(waist), planes, 0.5, w, nullptr, s);
      }
      KernelScope k(plan, SHT_KIND_FFT_INVERSE, s);
      launch_inverse_unfold<T>(plan, kUnfoldScalar, w, nullptr, planes, MP(grid), nullptr, s);
    });
  });
}

// ------------------------------------------------------------------ tuning
int sht_plan_set_tuning(sht_plan* plan, int key, int value) {
  return guarded([&] {
    check_transform_plan(plan);
    switch (key) {
      case SHT_TUNE_CONTRACTION:
        SHT_REQUIRE(value == 0 || value == 1, "SHT_TUNE_CONTRACTION is 0 or 1");
        SHT_REQUIRE(value == 0 || plan->prec == SHT_PREC_SPLIT16,
                    "SHT_TUNE_CONTRACTION = 1 applies to split16 plans");
        plan->tune_contraction = value;
        break;
      case SHT_TUNE_FFT:
        SHT_REQUIRE(value == 0 || value == 1, "SHT_TUNE_FFT is 0 or 1");
        if (value == 0) {
          SHT_REQUIRE(fast_fft_supported(plan),
                      "the register-resident FFT does not cover this grid or precision");
          if (!plan->fast_fft) fast_fft_init_constants(nullptr);
          plan->fast_fft = true;
        } else {
          plan->fast_fft = false;
        }
        break;
      case SHT_TUNE_TILE_ORDER:
        SHT_REQUIRE(value == 0 || value == 1, "SHT_TUNE_TILE_ORDER is 0 or 1");
        plan->tune_tile_order = value;
        break;
      case SHT_TUNE_TC_CTAS:
        SHT_REQUIRE(value >= 0 && value <= 4096, "SHT_TUNE_TC_CTAS is in [0, 4096]");
        plan->tune_tc_ctas = value;
        break;
      case SHT_TUNE_ACCUMULATORS:
        SHT_REQUIRE(value >= 0 && value <= 2, "SHT_TUNE_ACCUMULATORS is 0, 1 or 2");
        plan->tune_accumulators = value;
        break;
      case SHT_TUNE_SIMT_TILE:
        SHT_REQUIRE(value == 0 || value == 1, "SHT_TUNE_SIMT_TILE is 0 or 1");
        SHT_REQUIRE(value == 0 || plan->prec != SHT_PREC_F64,
                    "SHT_TUNE_SIMT_TILE 1 (64-wide column tiles) is an FP32 tile shape");
        plan->tune_simt_tile = value;
        break;
      default:
        throw Error{SHT_ERR_ARG, "unknown tuning key"};
    }
  });
}

int sht_plan_get_tuning(sht_plan* plan, int key, int* value) {
  return guarded([&] {
    check_transform_plan(plan);
    check_ptr(value, "value");
    switch (key) {
      case SHT_TUNE_CONTRACTION: *value = plan->tune_contraction; break;
      case SHT_TUNE_FFT: *value = plan->fast_fft ? 0 : 1; break;
      case SHT_TUNE_TILE_ORDER: *value = plan->tune_tile_order; break;
      case SHT_TUNE_TC_CTAS: *value = plan->tune_tc_ctas; break;
      case SHT_TUNE_ACCUMULATORS: *value = plan->tune_accumulators; break;
      case SHT_TUNE_SIMT_TILE: *value = plan->tune_simt_tile; break;
      default: throw Error{SHT_ERR_ARG, "unknown tuning key"};
    }
  });
}

}  // extern "C"
