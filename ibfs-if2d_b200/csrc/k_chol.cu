// k_chol.cu -- FP64 Cholesky factor, inverse factor and per-step solve of the
// stationary-body force system (operators.f90:766-819).
//
// Factor: one CTA per case runs choldc's column loop; each thread owns one
// row j and forms its dot product sequentially in the reference's descending
// k order with unfused multiply/subtract, so the factor matches choldc bit
// for bit given the same A. The factor is kept in the reference layout
// (cholmat strict lower triangle + cholvec), which is also the .chd layout.
// Solve: fb = L^-T (L^-1 rhsf) as two triangular GEMVs over an explicit
// inverse factor (one warp per row, coalesced row reads); the two halves read
// 8*Nf^2 bytes per step.
#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"

namespace ibfs {

__global__ void __launch_bounds__(1024) k_chol_factor(const DevCase* __restrict__ cases, const int* __restrict__ cids,
                                                      int* status) {
  const DevCase& C = cases[cids[blockIdx.x]];
  const int nf = C.nf;
  double* A = C.chol;             // cholmat(i,j) at (i-1) + (j-1)*nf
  double* vec = C.chol + (size_t)nf * nf;  // cholvec
  __shared__ int failed;
  if (threadIdx.x == 0) failed = 0;
  __syncthreads();
  for (int i = 1; i <= nf; i++) {
    // diagonal first (j = i), then the rest of the row range in parallel
    if (threadIdx.x == 0) {
      double sum = A[(i - 1) + (size_t)(i - 1) * nf];
      for (int k = i - 1; k >= 1; k--) {
        double p = __dmul_rn(A[(i - 1) + (size_t)(k - 1) * nf], A[(i - 1) + (size_t)(k - 1) * nf]);
        sum = __dsub_rn(sum, p);
      }
      if (!(sum > 0.0)) failed = 1;
      vec[i - 1] = sqrt(sum > 0.0 ? sum : 1.0);
    }
    __syncthreads();
    if (failed) break;
    double piv = vec[i - 1];
    for (int j = i + 1 + threadIdx.x; j <= nf; j += blockDim.x) {
      double sum = A[(i - 1) + (size_t)(j - 1) * nf];
      for (int k = i - 1; k >= 1; k--) {
        double p = __dmul_rn(A[(i - 1) + (size_t)(k - 1) * nf], A[(j - 1) + (size_t)(k - 1) * nf]);
        sum = __dsub_rn(sum, p);
      }
      A[(j - 1) + (size_t)(i - 1) * nf] = sum / piv;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && failed) atomicOr(status, 1);
}

// Linv = L^-1 (row-major), LinvT = its transpose (row-major), row by row:
// Linv[r][c] = (delta_rc - sum_{k=c}^{r-1} L[r][k] Linv[k][c]) / L[r][r].
__global__ void __launch_bounds__(1024) k_chol_inverse(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.x]];
  const int nf = C.nf;
  const double* A = C.chol;
  const double* vec = C.chol + (size_t)nf * nf;
  double* Li = C.Linv;
  double* LiT = C.LinvT;
  for (int r = 0; r < nf; r++) {
    double dr = vec[r];
    for (int c = threadIdx.x; c < nf; c += blockDim.x) {
      double v = 0.0;
      if (c <= r) {
        double s = (c == r) ? 1.0 : 0.0;
        for (int k = c; k < r; k++) s -= A[r + (size_t)k * nf] * Li[(size_t)k * nf + c];
        v = s / dr;
      }
      Li[(size_t)r * nf + c] = v;
      LiT[(size_t)c * nf + r] = v;
    }
    __syncthreads();
  }
}

// y = Linv * b (lower), then x = LinvT * y (upper); warp per row.
__global__ void k_tri_gemv(const DevCase* __restrict__ cases, const int* __restrict__ cids, int upper) {
  const DevCase& C = cases[cids[blockIdx.y]];
  const int nf = C.nf;
  int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  int lane = threadIdx.x & 31;
  if (row >= nf) return;
  const double* M = upper ? C.LinvT : C.Linv;
  const double* in = upper ? C.fwork : C.rhsf;
  double* out = upper ? C.fb : C.fwork;
  int k0 = upper ? row : 0, k1 = upper ? nf : row + 1;
  const double* Mr = M + (size_t)row * nf;
  double s = 0.0;
  for (int k = k0 + lane; k < k1; k += 32) s = fma(Mr[k], in[k], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[row] = s;
}

void launch_chol_factor(const DevCase* cases, const int* cids, int ncases, int* status, cudaStream_t st) {
  if (ncases) k_chol_factor<<<ncases, 1024, 0, st>>>(cases, cids, status);
}
void launch_chol_inverse(const DevCase* cases, const int* cids, int ncases, cudaStream_t st) {
  if (ncases) k_chol_inverse<<<ncases, 1024, 0, st>>>(cases, cids);
}
void launch_chol_solve(const DevCase* cases, const int* cids, int ncases, int max_nf, cudaStream_t st) {
  if (!ncases) return;
  dim3 g((max_nf + 7) / 8, ncases);
  k_tri_gemv<<<g, 256, 0, st>>>(cases, cids, 0);
  k_tri_gemv<<<g, 256, 0, st>>>(cases, cids, 1);
}

}  // namespace ibfs
