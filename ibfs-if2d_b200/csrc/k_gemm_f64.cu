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
//
// Split-K variants (SPLIT = 2 or 4) fill the machine when a launch group has
// few tiles (one case's 399^2 or 511^2 transform has 49-169 tiles for 148
// SMs): the SPLIT thread blocks of a cluster share one output tile, each
// summing a contiguous share of K; rank 0 adds the other ranks' partial tiles
// from their shared memory (distributed shared memory) in rank order, then
// applies the epilogue. The result is deterministic; it differs from the
// unsplit sum only in the order of the K partial sums.
#include <cooperative_groups.h>

#include <mutex>

#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"

namespace cg = cooperative_groups;

namespace ibfs {

constexpr int kBK = 16;

template <int BM, int BN, bool DUAL, int SPLIT>
__global__ void __launch_bounds__(256) k_gemm_f64(const GemmDesc* __restrict__ descs) {
  const GemmDesc& d = descs[blockIdx.y];
  const int tiles_m = (d.M + BM - 1) / BM;
  const int tiles_n = (d.N + BN - 1) / BN;
  const int tile = (int)blockIdx.x / SPLIT, rank = (int)blockIdx.x % SPLIT;
  // a cluster's blocks share a tile; all of them (or none) pass this test
  if (tile >= tiles_m * tiles_n) return;
  const int m0 = (tile % tiles_m) * BM, n0 = (tile / tiles_m) * BN;
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

  // this block's K blocks: all of them, or a contiguous share of the split
  const int nk_all = (K + kBK - 1) / kBK;
  const int per = (nk_all + SPLIT - 1) / SPLIT;
  const int kt0 = SPLIT > 1 ? min(nk_all, rank * per) : 0;
  const int nk = SPLIT > 1 ? min(nk_all, kt0 + per) : nk_all;
  if (kt0 < nk) {
    load(kt0 * kBK);
    store(0);
  }
  __syncthreads();
  for (int kt = kt0; kt < nk; kt++) {
    const int buf = (kt - kt0) & 1;
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

  if (SPLIT > 1) {
    // partial tiles through distributed shared memory, summed by rank 0 in
    // rank order (the main loop's last __syncthreads freed the operand tiles)
    double* part = smem;  // [TM*TN (x2 for DUAL)][256], thread-major per element
    constexpr int NP = TM * TN;
#pragma unroll
    for (int a = 0; a < TM; a++)
#pragma unroll
      for (int b = 0; b < TN; b++) {
        part[(a * TN + b) * 256 + tid] = acc[a][b];
        if (DUAL) part[(NP + a * TN + b) * 256 + tid] = acc2[DUAL ? a : 0][DUAL ? b : 0];
      }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    if (rank == 0) {
#pragma unroll 1
      for (int r = 1; r < SPLIT; r++) {
        const double* rp = cl.map_shared_rank(part, r);
#pragma unroll
        for (int a = 0; a < TM; a++)
#pragma unroll
          for (int b = 0; b < TN; b++) {
            acc[a][b] += rp[(a * TN + b) * 256 + tid];
            if (DUAL) acc2[DUAL ? a : 0][DUAL ? b : 0] += rp[(NP + a * TN + b) * 256 + tid];
          }
      }
    }
    cl.sync();  // the other ranks keep their shared memory until rank 0 has read it
    if (rank != 0) return;
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

template <int BM, int BN, bool DUAL, int SPLIT>
static size_t smem_bytes() {
  const size_t ops = 2 * kBK * BM + 2 * kBK * (BN + 1) * (DUAL ? 2 : 1);
  const size_t part = SPLIT > 1 ? (size_t)BM * BN * (DUAL ? 2 : 1) : 0;  // partial tiles of the split
  return sizeof(double) * (ops > part ? ops : part);
}

template <int BM, int BN, bool DUAL, int SPLIT>
static void set_attr() {
  cudaFuncSetAttribute(k_gemm_f64<BM, BN, DUAL, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem_bytes<BM, BN, DUAL, SPLIT>());
}

// Tile configurations: 0 64x64, 1 32x32, 2 64x32, 3 32x64 (unsplit; all four
// give bit-identical results), 4 32x32 split in 2 along K, 5 64x64 split in 4,
// 6 32x32 split in 4.
struct F64Cfg {
  int bm, bn, split;
};
static const F64Cfg kF64Cfg[kGemmF64Cfgs] = {{64, 64, 1}, {32, 32, 1}, {64, 32, 1}, {32, 64, 1},
                                             {32, 32, 2}, {64, 64, 4}, {32, 32, 4}};

// Raise the dynamic shared-memory limit of every instantiation (once per
// process, before any stream capture; handles may be created from several
// host threads).
void gemm_f64_init() {
  static std::once_flag once;
  std::call_once(once, []() {
    set_attr<64, 64, true, 1>(); set_attr<64, 64, false, 1>();
    set_attr<32, 32, true, 1>(); set_attr<32, 32, false, 1>();
    set_attr<64, 32, true, 1>(); set_attr<64, 32, false, 1>();
    set_attr<32, 64, true, 1>(); set_attr<32, 64, false, 1>();
    set_attr<32, 32, true, 2>(); set_attr<32, 32, false, 2>();
    set_attr<64, 64, true, 4>(); set_attr<64, 64, false, 4>();
    set_attr<32, 32, true, 4>(); set_attr<32, 32, false, 4>();
  });
}

template <int BM, int BN, bool DUAL, int SPLIT>
static void launch_cfg(const GemmDesc* d, int ndesc, int max_tiles, cudaStream_t st) {
  const size_t sm = smem_bytes<BM, BN, DUAL, SPLIT>();
  dim3 g(max_tiles * SPLIT, ndesc);
  if (SPLIT == 1) {
    k_gemm_f64<BM, BN, DUAL, SPLIT><<<g, 256, sm, st>>>(d);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = SPLIT;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k_gemm_f64<BM, BN, DUAL, SPLIT>, d);
}

int gemm_tiles(int M, int N, int cfg) {
  const F64Cfg& c = kF64Cfg[cfg < 0 || cfg >= kGemmF64Cfgs ? 0 : cfg];
  return ((M + c.bm - 1) / c.bm) * ((N + c.bn - 1) / c.bn);
}

void launch_gemm_f64(const GemmDesc* d, int ndesc, int max_tiles, int cfg, bool dual, cudaStream_t st) {
  if (ndesc == 0) return;
  switch (cfg) {
    case 0: dual ? launch_cfg<64, 64, true, 1>(d, ndesc, max_tiles, st) : launch_cfg<64, 64, false, 1>(d, ndesc, max_tiles, st); break;
    case 1: dual ? launch_cfg<32, 32, true, 1>(d, ndesc, max_tiles, st) : launch_cfg<32, 32, false, 1>(d, ndesc, max_tiles, st); break;
    case 2: dual ? launch_cfg<64, 32, true, 1>(d, ndesc, max_tiles, st) : launch_cfg<64, 32, false, 1>(d, ndesc, max_tiles, st); break;
    case 3: dual ? launch_cfg<32, 64, true, 1>(d, ndesc, max_tiles, st) : launch_cfg<32, 64, false, 1>(d, ndesc, max_tiles, st); break;
    case 4: dual ? launch_cfg<32, 32, true, 2>(d, ndesc, max_tiles, st) : launch_cfg<32, 32, false, 2>(d, ndesc, max_tiles, st); break;
    case 5: dual ? launch_cfg<64, 64, true, 4>(d, ndesc, max_tiles, st) : launch_cfg<64, 64, false, 4>(d, ndesc, max_tiles, st); break;
    default: dual ? launch_cfg<32, 32, true, 4>(d, ndesc, max_tiles, st) : launch_cfg<32, 32, false, 4>(d, ndesc, max_tiles, st); break;
  }
}

}  // namespace ibfs
