// sht_forward_static_scratch: the grid -> spectral transform for callers that
// cannot allocate device memory at call time.
//
// Who needs it: code that runs where cudaMalloc is off limits -- inside a
// host callback or a custom allocator hook, under an external memory manager
// that owns the whole device budget, or on a path that must never block on
// the driver's allocator -- can create its plan once at start-up and then
// transform through this entry point without any further allocation.  The
// regular sht_forward grows the plan's scratch on demand instead.
//
// The scratch (the equator-folded Fourier waist and the folded analysis
// output) lives in one file-scope device array of SHT_STATIC_SCRATCH_BYTES.
// Every GPU that loads the library holds that array until the process exits.
// In host code the array's name is only a stand-in for the symbol, so its
// device address is looked up with cudaGetSymbolAddress once per device, the
// first time the entry point runs with that device current; that first call
// should therefore happen before any stream capture.  All calls share the
// one array: calls that overlap on the GPU (on different streams, or from
// different threads) race on it.  Nothing in it has to start at zero: each
// call writes every element it later reads.
#include <mutex>

#include "sht_plan.h"

namespace {

__device__ __align__(256) unsigned char g_static_scratch[SHT_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Device address of g_static_scratch on the current device (looked up once).
void* scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices)
    throw sht::Error{SHT_ERR_ARG, "device ordinal out of range for the static scratch table"};
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_addr[device] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw sht::Error{SHT_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") +
                                         cudaGetErrorString(e)};
    g_scratch_addr[device] = p;
  }
  return g_scratch_addr[device];
}

template <typename T>
void forward_static(sht_plan* p, const T* grid, int64_t planes, T* coeff, void* base,
                    cudaStream_t s) {
  const int64_t R = 2 * planes;
  T* w = static_cast<T*>(base);
  const int64_t w_bytes = sht::round_up((int64_t)sizeof(T) * p->wfold_elems(R), 256);
  T* c = reinterpret_cast<T*>(static_cast<unsigned char*>(base) + w_bytes);
  sht::launch_forward_fold<T>(p, grid, nullptr, planes, w, s);
  sht::launch_gemm_simt<T>(p, 1, 0, static_cast<const T*>(p->analysis), w, c, R, s);
  sht::launch_unpack<T>(p, sht::kUnpackScalar, c, nullptr, planes, coeff, nullptr, s);
}

}  // namespace

extern "C" int sht_forward_static_scratch(sht_plan* plan, const void* grid, int64_t planes,
                                          void* coeff, void* stream) {
  try {
    sht::clear_error();
    if (plan == nullptr) throw sht::Error{SHT_ERR_ARG, "plan is NULL"};
    if (plan->geometry_only || plan->basis == nullptr)
      throw sht::Error{SHT_ERR_ARG, "plan cannot transform (geometry-only or not built)"};
    if (planes < 0) throw sht::Error{SHT_ERR_ARG, "planes must be >= 0"};
    if (planes == 0) return SHT_OK;
    if (grid == nullptr || coeff == nullptr) throw sht::Error{SHT_ERR_ARG, "grid or coeff is NULL"};
    if (plan->prec == SHT_PREC_SPLIT16)
      throw sht::Error{SHT_ERR_ARG,
                       "sht_forward_static_scratch serves SHT_PREC_F32 and SHT_PREC_F64 plans; "
                       "the split-FP16 contraction builds per-call work lists"};
    int device = 0;
    SHT_CUDA_OR_THROW(cudaGetDevice(&device));
    if (device != plan->device)
      throw sht::Error{SHT_ERR_ARG, "the current device is not the plan's device"};
    const int64_t R = 2 * planes;
    const int64_t elem = (int64_t)plan->elem();
    const int64_t need = sht::round_up(elem * plan->wfold_elems(R), 256) + elem * plan->cfold_elems(R);
    if (need > (int64_t)SHT_STATIC_SCRATCH_BYTES) {
      const int64_t per_plane = sht::round_up(elem * plan->wfold_elems(2), 256) + elem * plan->cfold_elems(2);
      throw sht::Error{SHT_ERR_ARG,
                       "sht_forward_static_scratch: " + std::to_string(planes) + " planes need " +
                           std::to_string(need) + " bytes of scratch, above the fixed " +
                           std::to_string((int64_t)SHT_STATIC_SCRATCH_BYTES) +
                           " bytes; at most about " +
                           std::to_string((int64_t)SHT_STATIC_SCRATCH_BYTES / per_plane) +
                           " planes per call for this plan"};
    }
    void* base = scratch_address(device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (plan->prec == SHT_PREC_F64)
      forward_static<double>(plan, static_cast<const double*>(grid), planes,
                             static_cast<double*>(coeff), base, s);
    else
      forward_static<float>(plan, static_cast<const float*>(grid), planes,
                            static_cast<float*>(coeff), base, s);
    return SHT_OK;
  } catch (const sht::Error& e) {
    sht::set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    sht::set_error(e.what());
    return SHT_ERR_STATE;
  }
}
