// k_precision.cu -- split-precision (3xBF16 tcgen05) transforms + FP64 refinement.
#include "ibfs_precision.cuh"

namespace ibfs {

struct PrecisionPlan {
  int dummy;
};

static const char* g_perr = "split-precision form not built";

int precision_init(PrecisionPlan*& pp, cudaStream_t, const std::vector<DevCase>&, const DevCase*, Alloc) {
  pp = nullptr;
  return 7;
}
void precision_free(PrecisionPlan* pp) { delete pp; }
const char* precision_error() { return g_perr; }
void build_precision_step1(PrecisionPlan*, Prog&, const DevCase*, const std::vector<DevCase>&, cudaStream_t) {}
void build_precision_vort2flux(PrecisionPlan*, Prog&, const DevCase*, const std::vector<DevCase>&,
                               const std::vector<int>&, bool, cudaStream_t) {}
void build_precision_ainv(PrecisionPlan*, Prog&, const DevCase*, const std::vector<DevCase>&, int, cudaStream_t) {}
int precision_apply_op(PrecisionPlan*, int, const DevCase*, const DevCase&, cudaStream_t) { return 7; }

}  // namespace ibfs
