// Split-precision tensor-core Legendre contraction (tcgen05): placeholder
// until the kernel is built; SPLIT16 plans use the FP32 SIMT kernel.
#include "sht_plan.h"

namespace sht {

void build_tc_tables(sht_plan* p, const double*, const double*, const double*, const double*,
                     const double*, cudaStream_t) {
  p->tc = nullptr;
}

void destroy_tc_tables(sht_plan* p) { p->tc = nullptr; }

void launch_gemm_tc(const sht_plan*, int, int, int, const float*, float*, int64_t, cudaStream_t) {
  throw Error{SHT_ERR_STATE, "tensor-core contraction not available"};
}

}  // namespace sht
