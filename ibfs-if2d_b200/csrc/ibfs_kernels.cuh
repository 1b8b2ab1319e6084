// ibfs_kernels.cuh -- launchers of the B200 IBFS kernels (host-callable).
#pragma once
#include <functional>
#include <vector>

#include "ibfs_common.cuh"

namespace ibfs {

// One launch (or a fixed pair of launches) of the step program, with its
// class for profiling and its algorithmic flops.
enum ProgTag { TAG_STENCIL = 0, TAG_GEMM_F64 = 1, TAG_GEMM_TC = 2, TAG_CHOL = 3, TAG_SPLIT = 4, TAG_NTAGS = 5 };
struct ProgEntry {
  std::function<void()> fn;
  int tag;
  double flops;
};
using Prog = std::vector<ProgEntry>;

// Dense-GEMM sine transform (one half of a 2-D DST-I, myfft.f90:83-94):
//   C(M x N) = A(M x K) * B(K x N), column-major, FP64, with fused prologue
//   (apply_bc of a coarser streamfunction, operators.f90:231-233) and
//   epilogues for the spectral scalings of ctci / ainv / the CN update.
enum GemmPro { PRO_NONE = 0, PRO_APPLY_BC = 1 };
enum GemmEpi {
  EPI_STORE = 0,     // C = acc
  EPI_LAMINV = 1,    // C = laminv .* acc                    (ctci, myfft.f90:106)
  EPI_AINV = 2,      // C = lam1i(:,:,1) .* acc / normalize  (ainv, myfft.f90:121)
  EPI_CN = 3,        // C = lam1i_k .* (acc + lam1_k .* acc2)  (operators.f90:126-130)
  EPI_SUBTRACT = 4,  // C = C - acc                          (operators.f90:174)
  EPI_ADD = 5,       // C = C + acc                          (adjoint accumulation)
  EPI_ADJ_CN = 6,    // C = lam1i_k .* acc, C2 = lam1i_k .* lam1_k .* acc (adjoint of the CN update)
};

struct GemmDesc {
  const double* A;
  const double* B;
  const double* B2;  // second right operand (EPI_CN)
  double* C;
  double* C2;  // second output (EPI_ADJ_CN)
  int M, N, K, lda, ldb, ldc;
  int pro, epi;
  int m, n, k;             // grid of the node field and its level
  const double* bcsrc;     // PRO_APPLY_BC: coarser-level streamfunction
  const double* cosx;      // cos(pi i/m), i=1..m-1
  const double* cosy;      // cos(pi j/n), j=1..n-1
  double dt, re, del22, norm;
};

// tile_cfg 0..3: unsplit tiles (bit-identical results); 4..6: split-K over a
// cluster of 2 or 4 blocks (kGemmF64Cfgs configurations in all)
constexpr int kGemmF64Cfgs = 7;
void launch_gemm_f64(const GemmDesc* d_descs, int ndesc, int max_tiles, int tile_cfg, bool dual, cudaStream_t st);
int gemm_tiles(int M, int N, int tile_cfg);
void gemm_f64_init();

void launch_lastbc(const DevCase* cases, const LevelItem* items, int nitems, int max_ring, cudaStream_t st);
// Grouped element-wise launches: block b of a launch covers elements
// [map[b].y, map[b].y + kBlockElems) of item map[b].x (block_map(counts)).
constexpr int kBlockElems = 1024;
std::vector<int2> block_map(const std::vector<int>& counts);
// interior nodes coarsify writes on level k > 1 (operators.f90:307-333)
__host__ __device__ inline int coarsify_count(int m, int n) {
  return (3 * m / 4 - (m / 4 + 2) + 1) * (3 * n / 4 - (n / 4 + 2) + 1);
}
void launch_vertex(const DevCase* cases, int c, int k, int ns, double* out, cudaStream_t st);
void launch_rhs(const DevCase* cases, const LevelItem* items, const int2* bmap, int nblocks, int first,
                cudaStream_t st);
// Split-precision level update input (k_rhs_split): per (case, level) item,
// b = scale * rhsA + (omega_k - nu C^T C omega_k) into b64 (FP64, column-major)
// and three BF16 slices Xs [slice][i][j] (row stride ld, slice stride sX).
struct RhsSplitDesc {
  double scale, nu;
  double* b64;
  uint16_t* Xs;
  long long sX;
  int ld;
};
// one block per 32 x 32 node tile: bmap[b] = {item, tile}, tiles i-fastest
void launch_rhs_split(const DevCase* cases, const LevelItem* items, const RhsSplitDesc* sd, const int2* bmap,
                      int nblocks, int first, cudaStream_t st);
void launch_coarsify(const DevCase* cases, const LevelItem* items, const int2* bmap, int nblocks, cudaStream_t st);
void launch_curl(const DevCase* cases, const LevelItem* items, const int2* bmap, int nblocks, cudaStream_t st);
void launch_regrot(const DevCase* cases, const int* cids, const int2* bmap, int nblocks, cudaStream_t st);
void launch_rhsf(const DevCase* cases, const int* cids, int ncases, int max_nf, cudaStream_t st);
void launch_regT_out(const DevCase* cases, const int* cids, int ncases, int max_nf, double* const* outs,
                     cudaStream_t st);
void launch_unit_fb(const DevCase* cases, const int* cids, const int* cols, int ncases, int max_nf, cudaStream_t st);
void launch_outputs(const DevCase* cases, const LevelItem* items, int nitems, const int* cids, const int* item_base,
                    int ncases, double* partial, cudaStream_t st);
void launch_step_begin(const DevCase* cases, int ncases, cudaStream_t st);

// Moving body and CG (grid.f90:523-576, 142-230; operators.f90:393-441).
void launch_move_body(const DevCase* cases, const int* cids, int ncases, int max_nb, cudaStream_t st);
void launch_actuate(const DevCase* cases, const int* cids, int ncases, int max_nact, cudaStream_t st);
void launch_setup_reg_moving(const DevCase* cases, const int* cids, int ncases, int max_nf, int max_patch,
                             cudaStream_t st);
void launch_cg_start(const DevCase* cases, const int* cids, int ncases, cudaStream_t st);
void launch_cg_alpha(const DevCase* cases, const int* cids, int ncases, int recompute, cudaStream_t st);
void launch_cg_resid(const DevCase* cases, const int* cids, int ncases, cudaStream_t st);
void launch_cg_beta(const DevCase* cases, const int* cids, int ncases, cudaStream_t st);

// Cholesky factor / inverse / solve (operators.f90:766-819).
void launch_chol_factor(const DevCase* cases, const int* cids, int ncases, int* status, cudaStream_t st);
void launch_chol_inverse(const DevCase* cases, const int* cids, int ncases, cudaStream_t st);
void launch_chol_solve(const DevCase* cases, const int* cids, int ncases, int max_nf, cudaStream_t st);

}  // namespace ibfs
