// k_gemm_f64.cu -- FP64 dense sine-matrix transforms for the plain method.
//
// A 2-D DST-I of an (m-1)x(n-1) field X (FFTW RODFT00 in both directions,
// myfft.f90:83-94) is Y = S_m X S_n with S_N(a,b) = 2 sin(pi a b / N). Each
// half is one column-major GEMM: T = X*S_n ("right") and Y = S_m*T ("left").
// The spectral scalings of ctci / ainv / the Crank-Nicolson update and the
// edge boundary terms of vort2flux are fused into the epilogue / prologue.
//
// Register-tiled DFMA kernel: 256 threads, BMxBN tile, BK=16, each thread a
// (BM/16)x(BN/16) micro-tile on a strided lattice (conflict-free shared loads),
// double-buffered shared memory with register prefetch. Grouped: blockIdx.y
// selects a GemmDesc, blockIdx.x a tile of it.
#include <mutex>

#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"

namespace ibfs {

constexpr int kBK = 16;

template <int BM, int BN, bool DUAL>
__global__ void __launch_bounds__(256) k_gemm_f64(const GemmDesc* __restrict__ descs) {
  const GemmDesc& d = descs[blockIdx.y];
  const int tiles_m = (d.M + BM - 1) / BM;
  const int tiles_n = (d.N + BN - 1) / BN;
  if ((int)blockIdx.x >= tiles_m * tiles_n) return;
  const int m0 = (blockIdx.x % tiles_m) * BM, n0 = (blockIdx.x / tiles_m) * BN;
  constexpr int TM = BM / 16, TN = BN / 16;
  constexpr int A_PER = BM * kBK / 256, B_PER = kBK * BN / 256;
  constexpr int LDB = BN + 1;
  extern __shared__ double smem[];
  double* As = smem;                      // [2][BK][BM]
  double* Bs = As + 2 * kBK * BM;         // [2][BK][LDB]
  double* B2s = Bs + 2 * kBK * LDB;       // [2][BK][LDB] (DUAL)
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int M = d.M, N = d.N, K = d.K, lda = d.lda, ldb = d.ldb;
  const double* __restrict__ A = d.A;
  const double* __restrict__ B = d.B;
  const double* __restrict__ B2 = d.B2;
  const int pro = d.pro, gm = d.m, gn = d.n;
  const double* __restrict__ bcs = d.bcsrc;

  double acc[TM][TN], acc2[DUAL ? TM : 1][DUAL ? TN : 1];
#pragma unroll
  for (int a = 0; a < TM; a++)
#pragma unroll
    for (int b = 0; b < TN; b++) acc[a][b] = 0.0;
  if (DUAL) {
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) acc2[DUAL ? a : 0][DUAL ? b : 0] = 0.0;
  }
  double ra[A_PER], rb[B_PER], rb2[DUAL ? B_PER : 1];

  auto load = [&](int k0) {
#pragma unroll
    for (int e = 0; e < A_PER; e++) {
      int idx = tid + 256 * e, r = idx % BM, kk = idx / BM;
      int gr = m0 + r, gk = k0 + kk;
      double v = 0.0;
      if (gr < M && gk < K) {
        v = A[gr + (size_t)gk * lda];
        if (pro == PRO_APPLY_BC) {
          int a = gr + 1, b = gk + 1;
          if (a == 1 || a == gm - 1 || b == 1 || b == gn - 1)
            v = apply_bc_at(v, a, b, gm, gn, 1.0,
                            [&](int side, int I) { return getbc_raw(bcs, gm, gn, side, I) * 1.0; });
        }
      }
      ra[e] = v;
    }
#pragma unroll
    for (int e = 0; e < B_PER; e++) {
      int idx = tid + 256 * e, kk = idx % kBK, c = idx / kBK;
      int gk = k0 + kk, gc = n0 + c;
      bool ok = gk < K && gc < N;
      rb[e] = ok ? B[gk + (size_t)gc * ldb] : 0.0;
      if (DUAL) rb2[DUAL ? e : 0] = ok ? B2[gk + (size_t)gc * ldb] : 0.0;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int e = 0; e < A_PER; e++) {
      int idx = tid + 256 * e, r = idx % BM, kk = idx / BM;
      As[(buf * kBK + kk) * BM + r] = ra[e];
    }
#pragma unroll
    for (int e = 0; e < B_PER; e++) {
      int idx = tid + 256 * e, kk = idx % kBK, c = idx / kBK;
      Bs[(buf * kBK + kk) * LDB + c] = rb[e];
      if (DUAL) B2s[(buf * kBK + kk) * LDB + c] = rb2[DUAL ? e : 0];
    }
  };

  const int nk = (K + kBK - 1) / kBK;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < nk; kt++) {
    const int buf = kt & 1;
    if (kt + 1 < nk) load((kt + 1) * kBK);
    const double* as = As + buf * kBK * BM;
    const double* bs = Bs + buf * kBK * LDB;
    const double* bs2 = B2s + buf * kBK * LDB;
#pragma unroll
    for (int kk = 0; kk < kBK; kk++) {
      double av[TM], bv[TN];
#pragma unroll
      for (int a = 0; a < TM; a++) av[a] = as[kk * BM + tx + 16 * a];
#pragma unroll
      for (int b = 0; b < TN; b++) bv[b] = bs[kk * LDB + ty + 16 * b];
#pragma unroll
      for (int a = 0; a < TM; a++)
#pragma unroll
        for (int b = 0; b < TN; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
      if (DUAL) {
#pragma unroll
        for (int b = 0; b < TN; b++) bv[b] = bs2[kk * LDB + ty + 16 * b];
#pragma unroll
        for (int a = 0; a < TM; a++)
#pragma unroll
          for (int b = 0; b < TN; b++) acc2[DUAL ? a : 0][DUAL ? b : 0] = fma(av[a], bv[b], acc2[DUAL ? a : 0][DUAL ? b : 0]);
      }
    }
    if (kt + 1 < nk) store(buf ^ 1);
    __syncthreads();
  }

  // epilogue
  const int epi = d.epi;
  double* __restrict__ Cp = d.C;
  const int ldc = d.ldc;
#pragma unroll
  for (int a = 0; a < TM; a++) {
    int r = m0 + tx + 16 * a;
    if (r >= M) continue;
#pragma unroll
    for (int b = 0; b < TN; b++) {
      int c = n0 + ty + 16 * b;
      if (c >= N) continue;
      double x = acc[a][b];
      size_t o = r + (size_t)c * ldc;
      if (epi == EPI_STORE) {
        Cp[o] = x;
      } else if (epi == EPI_SUBTRACT) {
        Cp[o] = Cp[o] - x;
      } else if (epi == EPI_ADD) {
        Cp[o] = Cp[o] + x;
      } else {
        double lam = lam_ij(d.cosx[r], d.cosy[c]);
        if (epi == EPI_LAMINV) {
          Cp[o] = (1.0 / lam / d.norm) * x;
        } else if (epi == EPI_AINV) {
          double l1i = 1.0 / (1.0 + 0.5 * d.dt * lam / d.del22 / d.re);
          Cp[o] = l1i * x / d.norm;
        } else if (epi == EPI_ADJ_CN) {
          double nu = 0.5 * d.dt * lam / d.del22 / d.re;
          double l1 = (1.0 - nu) / d.norm;
          double l1i = 1.0 / (1.0 + nu);
          Cp[o] = l1i * x;
          d.C2[o] = l1i * l1 * x;
        } else {  // EPI_CN
          double nu = 0.5 * d.dt * lam / d.del22 / d.re;
          double l1 = (1.0 - nu) / d.norm;
          double l1i = 1.0 / (1.0 + nu);
          double x2 = DUAL ? acc2[DUAL ? a : 0][DUAL ? b : 0] : 0.0;
          Cp[o] = l1i * (x + l1 * x2);
        }
      }
    }
  }
}

template <int BM, int BN, bool DUAL>
static size_t smem_bytes() {
  return sizeof(double) * (2 * kBK * BM + 2 * kBK * (BN + 1) * (DUAL ? 2 : 1));
}

template <int BM, int BN, bool DUAL>
static void set_attr() {
  cudaFuncSetAttribute(k_gemm_f64<BM, BN, DUAL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem_bytes<BM, BN, DUAL>());
}

// Raise the dynamic shared-memory limit of every instantiation (once per
// process, before any stream capture; handles may be created from several
// host threads).
void gemm_f64_init() {
  static std::once_flag once;
  std::call_once(once, []() {
    set_attr<64, 64, true>(); set_attr<64, 64, false>();
    set_attr<32, 32, true>(); set_attr<32, 32, false>();
    set_attr<64, 32, true>(); set_attr<64, 32, false>();
    set_attr<32, 64, true>(); set_attr<32, 64, false>();
  });
}

template <int BM, int BN, bool DUAL>
static void launch_cfg(const GemmDesc* d, int ndesc, int max_tiles, cudaStream_t st) {
  size_t sm = smem_bytes<BM, BN, DUAL>();
  dim3 g(max_tiles, ndesc);
  k_gemm_f64<BM, BN, DUAL><<<g, 256, sm, st>>>(d);
}

int gemm_tiles(int M, int N, int cfg) {
  int bm = (cfg == 0 || cfg == 2) ? 64 : 32;
  int bn = (cfg == 0 || cfg == 3) ? 64 : 32;
  return ((M + bm - 1) / bm) * ((N + bn - 1) / bn);
}

void launch_gemm_f64(const GemmDesc* d, int ndesc, int max_tiles, int cfg, bool dual, cudaStream_t st) {
  if (ndesc == 0) return;
  switch (cfg) {
    case 0: dual ? launch_cfg<64, 64, true>(d, ndesc, max_tiles, st) : launch_cfg<64, 64, false>(d, ndesc, max_tiles, st); break;
    case 1: dual ? launch_cfg<32, 32, true>(d, ndesc, max_tiles, st) : launch_cfg<32, 32, false>(d, ndesc, max_tiles, st); break;
    case 2: dual ? launch_cfg<64, 32, true>(d, ndesc, max_tiles, st) : launch_cfg<64, 32, false>(d, ndesc, max_tiles, st); break;
    default: dual ? launch_cfg<32, 64, true>(d, ndesc, max_tiles, st) : launch_cfg<32, 64, false>(d, ndesc, max_tiles, st); break;
  }
}

}  // namespace ibfs
