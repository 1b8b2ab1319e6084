// k_static.cu -- 2-D DST-I of a device field that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a
// transform: a driver that hands every byte of device memory to its own pool
// manager up front, or a host language runtime that forbids the CUDA
// allocator on its solver thread. ibfs_dst2d_noalloc serves them. The
// caller passes device pointers to the input and output fields; the
// intermediate product of the two transform halves lives in the
// file-scope array below, and the sine coefficients are computed in the
// kernels, so no descriptor, table or work buffer is allocated.
//
// The transform is the reference's dst (myfft.f90:83-94, FFTW RODFT00 in
// both directions), Y = S_m X S_n with S_N(a,b) = 2 sin(pi a b / N), as two
// FP64 GEMM halves: T = X*S_n into the static scratch, then Y = S_m*T.
//
// Limits and sharing: m-1 and n-1 may not exceed kNoAllocMaxN (511), i.e.
// grids up to 512x512 cells; larger sizes are rejected with IBFS_ERR_ARG.
// The scratch is kNoAllocMaxN^2 doubles (2.09 MB) on every GPU that loads this
// library, held until the process exits. All calls on a device share it and
// it keeps the last call's contents; each call overwrites the whole region it
// reads, so nothing needs clearing. Calls that overlap on the GPU (different
// streams, or different host threads, at the same time) race on the scratch
// and must be serialised by the caller.
#include <mutex>
#include <string>

#include "../../include/ibfs_capi.h"
#include "ibfs_common.cuh"

namespace ibfs {

int set_error(int code, const char* msg);  // ibfs_capi.cu: message for ibfs_last_error(NULL)

constexpr int kNoAllocMaxN = 511;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxN * kNoAllocMaxN];

// S_N(a,b) = 2 sin(pi (a+1)(b+1) / N), the argument reduced mod 2N exactly.
__device__ __forceinline__ double sine_coef(int a, int b, int N) {
  long long p = ((long long)(a + 1) * (b + 1)) % (2 * N);
  return 2.0 * sinpi((double)p / (double)N);
}

// One half of the transform on a 32x32 output tile, 256 threads, BK = 16.
// LEFT: dst = S_m * src (src M x N, M = m-1); else dst = src * S_n.
template <bool LEFT>
__global__ void __launch_bounds__(256) k_dst_half_noalloc(const double* __restrict__ src, double* __restrict__ dst,
                                                          int m, int n) {
  const int M = m - 1, N = n - 1, K = LEFT ? M : N;
  const int tiles_m = (M + 31) / 32;
  const int m0 = (blockIdx.x % tiles_m) * 32, n0 = (blockIdx.x / tiles_m) * 32;
  __shared__ double As[16][32];
  __shared__ double Bs[16][33];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
    for (int e = 0; e < 2; e++) {
      int idx = tid + 256 * e;
      int r = idx % 32, kk = idx / 32;  // A tile (32 x 16)
      int gr = m0 + r, gk = k0 + kk;
      double a = 0.0;
      if (gr < M && gk < K) a = LEFT ? sine_coef(gr, gk, m) : src[gr + (size_t)gk * M];
      As[kk][r] = a;
      int kb = idx % 16, c = idx / 16;  // B tile (16 x 32)
      int gkb = k0 + kb, gc = n0 + c;
      double b = 0.0;
      if (gkb < K && gc < N) b = LEFT ? src[gkb + (size_t)gc * M] : sine_coef(gkb, gc, n);
      Bs[kb][c] = b;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; kk++) {
      double a0 = As[kk][tx], a1 = As[kk][tx + 16];
      double b0 = Bs[kk][ty], b1 = Bs[kk][ty + 16];
      acc[0][0] = fma(a0, b0, acc[0][0]);
      acc[0][1] = fma(a0, b1, acc[0][1]);
      acc[1][0] = fma(a1, b0, acc[1][0]);
      acc[1][1] = fma(a1, b1, acc[1][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; a++)
#pragma unroll
    for (int b = 0; b < 2; b++) {
      int r = m0 + tx + 16 * a, c = n0 + ty + 16 * b;
      if (r < M && c < N) dst[r + (size_t)c * M] = acc[a][b];
    }
}

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device. The array's
// name is only a host-side stand-in in host code, so the address is looked up
// once per device with that device current, on the first call there. The
// address is the one in the device's primary context (the CUDA runtime's);
// it is kept for the life of the process.
static int noalloc_scratch(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(IBFS_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_error(IBFS_ERR_ARG, "ibfs_dst2d_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(IBFS_ERR_CUDA, (std::string("ibfs_dst2d_noalloc: cudaGetSymbolAddress failed: ") +
                                       cudaGetErrorString(e)).c_str());
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return IBFS_OK;
}

}  // namespace ibfs

extern "C" int ibfs_dst2d_noalloc(const double* d_in, double* d_out, int m, int n, void* stream) {
  using namespace ibfs;
  if (!d_in || !d_out) return set_error(IBFS_ERR_ARG, "ibfs_dst2d_noalloc: null field pointer");
  if (m < 2 || n < 2 || m - 1 > kNoAllocMaxN || n - 1 > kNoAllocMaxN)
    return set_error(IBFS_ERR_ARG,
                     "ibfs_dst2d_noalloc: m-1 and n-1 must be in [1, 511] (grids up to 512x512 cells)");
  // An error left pending by earlier work on this thread stays the caller's:
  // refuse to launch rather than clear it and report it as this call's own.
  cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return set_error(IBFS_ERR_CUDA, (std::string("ibfs_dst2d_noalloc: an earlier CUDA error is pending: ") +
                                     cudaGetErrorString(pending)).c_str());
  double* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int M = m - 1, N = n - 1;
  int tiles = ((M + 31) / 32) * ((N + 31) / 32);
  k_dst_half_noalloc<false><<<tiles, 256, 0, st>>>(d_in, scratch, m, n);
  k_dst_half_noalloc<true><<<tiles, 256, 0, st>>>(scratch, d_out, m, n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(IBFS_ERR_CUDA, (std::string("ibfs_dst2d_noalloc launch: ") + cudaGetErrorString(e)).c_str());
  return IBFS_OK;
}
