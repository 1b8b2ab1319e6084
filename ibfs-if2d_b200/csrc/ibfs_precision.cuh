// ibfs_precision.cuh -- split-precision form of the sine transforms: each DST
// is a dense sine-matrix contraction on tcgen05 tensor cores with operands
// split into three BF16 slices (FP32 accumulation), and every solve that uses
// it gets one FP64 residual-correction sweep with the exact 5-point stencil.
#pragma once
#include <functional>
#include <vector>

#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"

namespace ibfs {

struct PrecisionPlan;
using Alloc = std::function<void*(size_t)>;

int precision_init(PrecisionPlan*& pp, cudaStream_t st, const std::vector<DevCase>& cases, const DevCase* d_cases,
                   Alloc alloc);
void precision_free(PrecisionPlan* pp);
// Limit (seconds, 0..60) of every bounded wait of the tensor-core GEMM;
// probe != 0 makes every block wait first on a barrier nothing completes.
int precision_set_wait_limit(PrecisionPlan* pp, double seconds, int probe);
// Tile configuration of the tensor-core GEMM: 1 (128x128, K blocks of 64, two
// stages), 2 (128x256, K 32, two stages), 3 (128x128, K 32, four stages), or 0
// for the measured autotuner.
void precision_set_tile(PrecisionPlan* pp, int cfg);
// Refinement: slices per operand of the correction solves (0 = three for the
// Poisson solves, two for the others; 2 or 3 = all) and correction sweeps of
// the Poisson (ctci) solves (1, the default, or 2).
void precision_set_refine(PrecisionPlan* pp, int slices, int poisson_sweeps);
// Configurations chosen for the GEMM launch groups built since the last reset.
const std::vector<int>& precision_tile_choices(const PrecisionPlan* pp);
void precision_reset_tile_choices(PrecisionPlan* pp);
const char* precision_error();
void build_precision_step1(PrecisionPlan* pp, Prog& P, const DevCase* dcases, const std::vector<DevCase>& cs,
                           cudaStream_t st);
void build_precision_vort2flux(PrecisionPlan* pp, Prog& P, const DevCase* dcases, const std::vector<DevCase>& cs,
                               const std::vector<int>& ids, bool curl_all, cudaStream_t st);
void build_precision_ainv(PrecisionPlan* pp, Prog& P, const DevCase* dcases, const std::vector<DevCase>& cs,
                          int final_epi, cudaStream_t st);
int precision_apply_op(PrecisionPlan* pp, int op, const DevCase* ds, const DevCase& s, cudaStream_t st);

}  // namespace ibfs
