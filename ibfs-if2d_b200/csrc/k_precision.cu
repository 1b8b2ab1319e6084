// k_precision.cu -- split-precision form of the IBFS sine transforms.
//
// Every Laplacian-type solve of the advance -- the Crank-Nicolson update
// (operators.f90:126-130), ctci in vort2flux (myfft.f90:97-109) and ainv in the
// projection (myfft.f90:112-124) -- inverts an operator that is diagonal in
// the 2-D DST-I basis. Here each DST half is a dense sine-matrix GEMM on the
// tcgen05 tensor cores with both operands split into three BF16 slices
// (x = x0 + x1 + x2, 8 significant bits each) and the six leading slice
// products accumulated in one FP32 TMEM tile. Each solve is followed by one
// FP64 residual-correction sweep with the exact 5-point stencil:
//     x0 = S f S v        r = v - A x0 (FP64)        x = x0 + S f S r
// which brings the ~1e-6 error of one split solve down to ~1e-12.
//
// GEMM kernel (k_gemm_tc_persist): a persistent launch over all 128x128
// output tiles of all (case, level) GEMMs of one stage, one CTA per SM. Per K
// block of 64 the six operand tiles (A0..A2, B0..B2, 96 KB) are brought into
// swizzled K-major shared memory by TMA (two stages, issued by one thread);
// one thread issues the slice products as tcgen05.mma (M128 N128 K16, BF16 in,
// FP32 accumulate in TMEM, double-buffered accumulators); eight warps drain
// them with tcgen05.ld. The 128-wide tile was measured against a 256-wide one
// with K blocks of 32 (38.8 vs 42.2 ms of GEMM per step of the 256-case batch)
// and kept. All mbarrier waits are bounded in time; a wait that gives up sets
// an error status, the CTA frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ibfs_precision.cuh"

namespace ibfs {

typedef __nv_bfloat16 bf16;

// ---------------------------------------------------------------------------
// PTX wrappers (sm_100a)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Default limit of every wait (a healthy wait lasts microseconds); the
// handle keeps the limit in device memory (ibfs_set_wait_limit), read once per
// CTA at kernel start.
constexpr uint64_t kWaitLimitNs = 1000000000ull;
// Limit of the waits that drain a CTA's own copies and products after a wait
// gave up; independent of the handle's limit so that the drain completes.
constexpr uint64_t kDrainLimitNs = 1000000000ull;

// Bounded wait for the phase with the given parity (try_wait may suspend the
// thread between polls); false once lim ns have passed since the first
// failed poll (with lim = 0: at the second failed poll).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t lim) {
  uint64_t t0 = 0;
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    const uint64_t t = global_ns();  // the clock is read only once a poll has failed
    if (t0 == 0) t0 = t;
    else if (t - t0 >= lim) return false;
  }
}

// Bounded spin without suspension, for the single producer / MMA threads whose
// waits sit on the critical path of every K block; false once lim ns have
// passed (the clock is read every 256 polls).
__device__ __forceinline__ bool mbar_spin(uint32_t bar, uint32_t parity, uint64_t lim) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255) {  // no clock read on the fast path
      const uint64_t t = global_ns();
      if (t0 == 0) t0 = t;
      else if (t - t0 >= lim) return false;
    }
  }
}

// A wait that gave up: flag the error (bit 2 of status[0]) and, for the first
// one, record where: status[1] = role (1 producer/stage free, 2 MMA/accumulator
// free, 3 MMA/stage loaded, 4 epilogue/accumulator ready), status[2] = block,
// status[3] = pipeline step; role 5 is the probe of the timeout test. A drain
// wait that gave up sets bit 4.
__device__ __forceinline__ void report_timeout(int* status, int role, int step) {
  atomicOr(status, 2);
  if (atomicCAS(status + 1, 0, role) == 0) {
    status[2] = (int)blockIdx.x;
    status[3] = step;
  }
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// K-major swizzled shared-memory matrix descriptor for rows of BK BF16:
// BK = 64 -> 128-byte rows, 128-byte swizzle (layout type 2), 8-row groups
// 1024 B apart; BK = 32 -> 64-byte rows, 64-byte swizzle (layout type 4),
// 8-row groups 512 B apart. LBO is unused for swizzled K-major; version 1.
template <int BK>
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((8 * BK * 2) >> 4) << 32;  // SBO
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)(BK == 64 ? 2 : 4) << 61;
  return d;
}

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M=128, N=BN.
template <int BN>
constexpr uint32_t idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((128u >> 4) << 24);
}

template <int BN>
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc_bf16<BN>()), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Split x into three BF16 slices (round to nearest each time).
__device__ __forceinline__ void split3(double x, bf16& s0, bf16& s1, bf16& s2) {
  s0 = __double2bfloat16(x);
  double r = x - (double)__bfloat162float(s0);
  s1 = __double2bfloat16(r);
  r = r - (double)__bfloat162float(s1);
  s2 = __double2bfloat16(r);
}

// ---------------------------------------------------------------------------
// Tensor-core GEMM
enum TcEpi { TC_SPLIT_COL = 0, TC_SCALE_SPLIT_ROW = 1, TC_F64_STORE = 2, TC_F64_ADD = 3 };
enum TcFactor { F_NONE = 0, F_LAMINV = 1, F_LAM1I_NORM = 2 };

// One GEMM of one (case, level) item. Operands are 3-slice BF16 arrays
// [slice][row][k] (k contiguous) described by TMA tensor maps; A rows are
// output rows, B rows output columns. K blocks of 64 (128-byte swizzle): mapA
// and mapB (boxes of 128 rows); K blocks of 32 (64-byte swizzle): mapA2 (128
// rows), mapB2 (256 rows) and mapB3 (128 rows).
struct __align__(64) TcDesc {
  CUtensorMap mapA;
  CUtensorMap mapB;
  CUtensorMap mapA2;
  CUtensorMap mapB2;
  CUtensorMap mapB3;
  int M, N, Kp;   // logical output extents; K padded to a multiple of 64
  int tiles_m;    // 128-row output tiles
  int nprod;      // slice products: 6 (three slices per operand) or 3 (two slices: A0B0 + A0B1 + A1B0)
  int epi, fkind;
  int ldcs, ldc;
  long long sC;
  bf16* Cs;       // split output: SPLIT_COL [j][i], SCALE_SPLIT_ROW [i][j]; 3 slices, stride sC
  double* C64;    // FP64 output, column-major, leading dimension ldc
  const float* lamx;  // 4 sin^2(pi (i+1) / 2m): eigenvalues of the 1-D 3-point Laplacian
  const float* lamy;
  float nu, norm;     // F_LAM1I_NORM: 1/((1 + nu lam) norm); F_LAMINV: 1/(lam norm)
};

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(dst),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

// Three-slice split of eight FP32 values (each slice the round-to-nearest
// BF16 of what the slices before it leave) with packed conversions: one
// cvt.rn.bf16x2.f32 rounds two values, and the packed words are the store
// format, so no repacking follows. u0, u1, u2: slices 0, 1, 2 of x[0..7].
__device__ __forceinline__ uint32_t cvt_bf16x2(float lo, float hi) {
  __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&p);
}
__device__ __forceinline__ float bf16lo(uint32_t p) { return __uint_as_float(p << 16); }
__device__ __forceinline__ float bf16hi(uint32_t p) { return __uint_as_float(p & 0xffff0000u); }
__device__ __forceinline__ void split8_packed(const float* x, uint4& u0, uint4& u1, uint4& u2) {
  uint32_t w0[4], w1[4], w2[4];
#pragma unroll
  for (int h = 0; h < 4; h++) {
    const float a = x[2 * h], b = x[2 * h + 1];
    w0[h] = cvt_bf16x2(a, b);
    const float ra = a - bf16lo(w0[h]), rb = b - bf16hi(w0[h]);
    w1[h] = cvt_bf16x2(ra, rb);
    w2[h] = cvt_bf16x2(ra - bf16lo(w1[h]), rb - bf16hi(w1[h]));
  }
  u0 = make_uint4(w0[0], w0[1], w0[2], w0[3]);
  u1 = make_uint4(w1[0], w1[1], w1[2], w1[3]);
  u2 = make_uint4(w2[0], w2[1], w2[2], w2[3]);
}

__device__ __forceinline__ void store4(bf16* dst, const bf16* v) {
  uint2 u;
  u.x = (uint32_t)__bfloat16_as_ushort(v[0]) | ((uint32_t)__bfloat16_as_ushort(v[1]) << 16);
  u.y = (uint32_t)__bfloat16_as_ushort(v[2]) | ((uint32_t)__bfloat16_as_ushort(v[3]) << 16);
  *reinterpret_cast<uint2*>(dst) = u;
}

// ---------------------------------------------------------------------------
// Persistent GEMM (k_gemm_tc_persist): one CTA per SM walks
// a cost-sorted work list of (desc, tile) items. Warp 0 lane 0 issues the TMA
// loads, warp 1 lane 0 the tcgen05.mma; the accumulator is double-buffered in
// TMEM (2 x BN columns) so warps 2-9 drain tile t (tcgen05.ld + epilogue)
// while tile t+1 is loaded and multiplied. Per-tile fixed costs (TMEM
// allocation, pipeline fill, epilogue) are thereby hidden behind the MMAs.
struct TcWork {
  int desc, tile;
};

// Tile configurations of the tensor-core GEMM (output tile 128 x BN, K blocks
// of BK, S pipeline stages of the three A and three B slice tiles), kTcCfgs of
// them:
//   1: BN 128, BK 64, 2 stages of 96 KB (128-byte rows, 128-byte swizzle)
//   2: BN 256, BK 32, 2 stages of 72 KB (64-byte rows, 64-byte swizzle)
//   3: BN 128, BK 32, 4 stages of 48 KB: the same tile as 1 with twice the
//      loads in flight ahead of the MMAs (three stages, ~2.3k cycles of MMA
//      at six products, against one stage of ~1.5k cycles in 1)
//   4: a 256 x 256 tile on a pair of CTAs (k_gemm_tc_pair), BK 64, 2 stages
//      of 96 KB per CTA
constexpr int kTcCfgs = 4;
template <int BN, int BK> constexpr int tc_ab() { return 128 * BK * 2; }  // one A slice tile
template <int BN, int BK> constexpr int tc_bb() { return BN * BK * 2; }   // one B slice tile
template <int BN, int BK> constexpr int tc_stage() { return 3 * tc_ab<BN, BK>() + 3 * tc_bb<BN, BK>(); }
constexpr int kPEpiWarps = 8;                                  // two warps per TMEM lane quarter
constexpr int kPThreads = 64 + 32 * kPEpiWarps;
constexpr int kPEpi = kPEpiWarps * 32 * 33 * 4;                // per-warp 32 x 33 FP32 staging
constexpr int kPBars = 256;                                    // barriers and the TMEM address slot
template <int BN, int BK, int S> constexpr int tc_smem() { return S * tc_stage<BN, BK>() + kPEpi + 1024 + kPBars; }
static_assert(tc_smem<128, 64, 2>() <= 232448, "persistent GEMM shared memory above the per-CTA limit");
static_assert(tc_smem<256, 32, 2>() <= 232448, "persistent GEMM shared memory above the per-CTA limit");
static_assert(tc_smem<128, 32, 4>() <= 232448, "persistent GEMM shared memory above the per-CTA limit");

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// Epilogue of chunks [c0, c1) (32 columns each) of one 128x128 tile for one
// warp: 32 rows starting at r0, this lane's row i = r0 + lane; trow = TMEM
// address of the warp's lanes at the accumulator; stg = the warp's 32 x 33
// FP32 staging area. Split outputs are restaged so that every warp store
// writes eight whole 64-byte row segments (lane L: segment L / 4 + 8 k, 16-byte
// part L % 4); FP64 outputs are column-major, so a warp store of one column
// is 32 consecutive doubles.
__device__ __forceinline__ void tc_epilogue(const TcDesc& d, int n0, uint32_t trow, int r0, int lane, float* stg,
                                            int c0, int c1) {
  const int M = d.M, N = d.N, epi = d.epi, fkind = d.fkind, ldcs = d.ldcs, ldc = d.ldc;
  const long long sC = d.sC;
  bf16* const Cs = d.Cs;
  double* const C64 = d.C64;
  const int i = r0 + lane;
  const int seg = lane >> 2, part = lane & 3;
  float lx = 0.f, nu = 0.f, norm = 1.f;
  const float* lamy = nullptr;
  if (epi == TC_SCALE_SPLIT_ROW) {
    lx = i < M ? __ldg(&d.lamx[i]) : 0.f;
    nu = d.nu;
    norm = d.norm;
    lamy = d.lamy;
  }
#pragma unroll 1
  for (int ch = c0; ch < c1; ch++) {
    float v[32];
    tmem_ld32(trow + ch * 32, v);
    const int jb = n0 + ch * 32;
    if (epi == TC_SPLIT_COL) {
      // output Cs[j][i] (i contiguous): stage column-major, then lane writes
      // column jb + seg + 8k, rows r0 + 8 part .. + 7
#pragma unroll
      for (int t = 0; t < 32; t++) stg[t * 33 + lane] = v[t];
      __syncwarp();
      if (r0 < ldcs) {
#pragma unroll 1
        for (int k = 0; k < 4; k++) {
          const int c = seg + 8 * k;
          float x[8];
#pragma unroll
          for (int e = 0; e < 8; e++) x[e] = stg[c * 33 + part * 8 + e];
          uint4 u0, u1, u2;
          split8_packed(x, u0, u1, u2);
          bf16* o = Cs + (size_t)(jb + c) * ldcs + r0 + part * 8;
          *reinterpret_cast<uint4*>(o) = u0;
          *reinterpret_cast<uint4*>(o + sC) = u1;
          *reinterpret_cast<uint4*>(o + 2 * sC) = u2;
        }
      }
      __syncwarp();
    } else if (epi == TC_SCALE_SPLIT_ROW) {
      // output Cs[i][j] (j contiguous): scale, stage row-major, then lane
      // writes row r0 + seg + 8k, columns jb + 8 part .. + 7
      const float ly = (jb + lane < N) ? __ldg(&lamy[jb + lane]) : 0.f;
#pragma unroll
      for (int t = 0; t < 32; t++) {
        const float lam = lx + __shfl_sync(0xffffffffu, ly, t);
        const float den = fkind == F_LAMINV ? lam * norm : (1.f + nu * lam) * norm;
        const bool in = i < M && jb + t < N;
        stg[lane * 33 + t] = in ? __fdividef(v[t], den) : 0.f;
      }
      __syncwarp();
      if (jb < ldcs) {
#pragma unroll 1
        for (int k = 0; k < 4; k++) {
          const int rr = seg + 8 * k;
          float x[8];
#pragma unroll
          for (int e = 0; e < 8; e++) x[e] = stg[rr * 33 + part * 8 + e];
          uint4 u0, u1, u2;
          split8_packed(x, u0, u1, u2);
          bf16* o = Cs + (size_t)(r0 + rr) * ldcs + jb + part * 8;
          *reinterpret_cast<uint4*>(o) = u0;
          *reinterpret_cast<uint4*>(o + sC) = u1;
          *reinterpret_cast<uint4*>(o + 2 * sC) = u2;
        }
      }
      __syncwarp();
    } else if (i < M) {
      if (epi == TC_F64_ADD) {
        // all loads first: a load after a store to the same array would
        // otherwise wait for it, one round trip per column
#pragma unroll
        for (int h = 0; h < 32; h += 16) {
          double old[16];
#pragma unroll
          for (int t = 0; t < 16; t++)
            old[t] = (jb + h + t < N) ? C64[(size_t)i + (size_t)(jb + h + t) * ldc] : 0.0;
#pragma unroll
          for (int t = 0; t < 16; t++)
            if (jb + h + t < N) C64[(size_t)i + (size_t)(jb + h + t) * ldc] = old[t] + (double)v[h + t];
        }
      } else {
#pragma unroll
        for (int t = 0; t < 32; t++)
          if (jb + t < N) C64[(size_t)i + (size_t)(jb + t) * ldc] = (double)v[t];
      }
    }
  }
}

template <int BN, int BK, int S>
__global__ void __launch_bounds__(kPThreads, 1) k_gemm_tc_persist(const TcDesc* __restrict__ descs,
                                                            const TcWork* __restrict__ work, int nwork,
                                                            int* __restrict__ status,
                                                            const unsigned long long* __restrict__ wait_ns) {
  constexpr int AB = tc_ab<BN, BK>(), BB = tc_bb<BN, BK>(), SB = tc_stage<BN, BK>();
  constexpr uint32_t TCOLS = 2 * BN;  // double-buffered FP32 accumulator columns
  static_assert((2 * S + 5) * 8 + 4 <= kPBars, "barrier area");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float* stg_all = reinterpret_cast<float*>(smem + S * SB);
  // full[S] empty[S] accf[2] acce[2] probe, then the TMEM address
  uint64_t* bars = (uint64_t*)(smem + S * SB + kPEpi);
  uint32_t* tmem_slot = (uint32_t*)(smem + S * SB + kPEpi + (2 * S + 5) * 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[S]);
  const uint32_t accf0 = smem_u32(&bars[2 * S]), acce0 = smem_u32(&bars[2 * S + 2]);
  const uint32_t probe = smem_u32(&bars[2 * S + 4]);
  const uint64_t lim = wait_ns[0];
  if (warp == 0) tmem_alloc(smem_u32(tmem_slot), TCOLS);
  if (tid == 0) {
    for (int b = 0; b < 2 * S + 2; b++) mbar_init(smem_u32(&bars[b]), 1);
    for (int b = 2 * S + 2; b < 2 * S + 4; b++) mbar_init(smem_u32(&bars[b]), kPEpiWarps);
    mbar_init(probe, 1);  // probe: nothing ever arrives on it
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int G = gridDim.x;
  bool to = false;
  // Test of the timeout path (wait_ns[1] != 0): before any copy or product is
  // issued, every role waits on the probe barrier, which nothing completes,
  // so each wait gives up after the limit and the block returns through the
  // same exit as a real timeout, with nothing in flight.
  if (wait_ns[1] != 0 && (tid == 0 || tid == 32 || warp >= 2)) {
    if (!mbar_wait(probe, 0, lim)) {
      report_timeout(status, 5, 0);
      to = true;
    }
  }

  if (tid == 0) {  // TMA producer
    int g = 0;
    for (int w = blockIdx.x; w < nwork && !to; w += G) {
      const TcDesc& d = descs[work[w].desc];
      const int tile = work[w].tile;
      const int m0 = (tile % d.tiles_m) * 128, n0 = (tile / d.tiles_m) * BN;
      const int nk = d.Kp / BK;
      const int ns = d.nprod == 3 ? 2 : 3;  // slices per operand
      const CUtensorMap* mA = BK == 64 ? &d.mapA : &d.mapA2;
      const CUtensorMap* mB = BK == 64 ? &d.mapB : (BN == 256 ? &d.mapB2 : &d.mapB3);
      for (int kb = 0; kb < nk; kb++, g++) {
        const int s = g % S;
        // stage s is free once the MMAs of load g - S completed (its empty phase (g - S) / S)
        if (g >= S && !mbar_spin(empty0 + 8 * s, ((g / S) + 1) & 1, lim)) { report_timeout(status, 1, g); to = true; break; }
        const uint32_t fb = full0 + 8 * s;
        mbar_expect_tx(fb, ns * (AB + BB));
        const uint32_t st = sbase + s * SB;
        for (int t = 0; t < ns; t++) tma_load_3d(st + t * AB, mA, kb * BK, m0, t, fb);
        for (int t = 0; t < ns; t++) tma_load_3d(st + 3 * AB + t * BB, mB, kb * BK, n0, t, fb);
      }
    }
    // Drain: only the last S stage loads can still be in flight (a stage is
    // reloaded only after the MMAs that read it completed, which waited for
    // its load). Their full-barrier phases complete when their bytes land;
    // in a run without timeouts they have completed already.
    for (int gi = g - 1; gi >= 0 && gi >= g - S; gi--)
      if (!mbar_spin(full0 + 8 * (gi % S), (gi / S) & 1, kDrainLimitNs)) atomicOr(status, 4);
  } else if (tid == 32) {  // MMA issuer
    constexpr int pa[6] = {0, 0, 1, 0, 1, 2};
    constexpr int pb[6] = {0, 1, 0, 2, 1, 0};
    // the stage ring ends below 2^18 bytes, so the 14-bit address field of
    // the descriptor never carries into the next field
    const uint64_t d0 = smem_desc_kmajor<BK>(sbase);
    int g = 0, t = 0;
    uint32_t last_bar = 0, last_par = 0;  // barrier and phase parity of the last commit
    for (int w = blockIdx.x; w < nwork && !to; w += G, t++) {
      const int a = t & 1, u = t >> 1;
      if (t >= 2 && !mbar_spin(acce0 + 8 * a, (u - 1) & 1, lim)) { report_timeout(status, 2, t); to = true; break; }
      tc_fence_after();
      const TcDesc& d = descs[work[w].desc];
      const int nk = d.Kp / BK;
      const int np = d.nprod == 3 ? 3 : 6;
      const uint32_t acc = tmem + a * BN;
      for (int kb = 0; kb < nk; kb++, g++) {
        const int s = g % S;
        if (!mbar_spin(full0 + 8 * s, (g / S) & 1, lim)) { report_timeout(status, 3, g); to = true; break; }
        tc_fence_after();
        // stage base descriptor; operand tiles and K steps are immediate
        // offsets (16-byte units) on its address field
        const uint64_t ds = d0 + (uint64_t)((uint32_t)(s * SB) >> 4);
#pragma unroll
        for (int p = 0; p < 6; p++) {
          if (p >= np) break;
#pragma unroll
          for (int k16 = 0; k16 < BK / 16; k16++)
            umma_bf16<BN>(acc, ds + (uint64_t)((pa[p] * AB + k16 * 32) >> 4),
                          ds + (uint64_t)((3 * AB + pb[p] * BB + k16 * 32) >> 4),
                          (kb > 0 || p > 0 || k16 > 0) ? 1u : 0u);
        }
        umma_commit(empty0 + 8 * s);
        last_bar = empty0 + 8 * s;
        last_par = (g / S) & 1;
      }
      if (!to) {
        umma_commit(accf0 + 8 * a);
        last_bar = accf0 + 8 * a;
        last_par = u & 1;
      }
    }
    // Drain: a commit's barrier phase completes once every MMA this thread
    // issued before it has completed; TMEM is freed only after that.
    if (last_bar && !mbar_spin(last_bar, last_par, kDrainLimitNs)) atomicOr(status, 4);
  } else if (warp >= 2) {  // epilogue warps
    const int q = warp & 3;                       // TMEM lane quarter this warp may access
    constexpr int CH = BN / 64;                   // 32-column chunks per warp
    const int c0 = ((warp - 2) >> 2) * CH;        // the warp's half of the tile's columns
    float* stg = stg_all + (warp - 2) * (32 * 33);
    int t = 0;
    for (int w = blockIdx.x; w < nwork && !to; w += G, t++) {
      const int a = t & 1, u = t >> 1;
      if (!mbar_wait(accf0 + 8 * a, u & 1, lim)) { report_timeout(status, 4, t); to = true; break; }
      tc_fence_after();
      const TcDesc& d = descs[work[w].desc];
      const int tile = work[w].tile;
      const int m0 = (tile % d.tiles_m) * 128, n0 = (tile / d.tiles_m) * BN;
      const int r0 = m0 + 32 * q;
      tc_epilogue(d, n0, tmem + a * BN + ((uint32_t)(32 * q) << 16), r0, lane, stg, c0, c0 + CH);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce0 + 8 * a);
    }
  }
  __syncwarp();
  __syncthreads_or(to);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TCOLS);
}

// ---------------------------------------------------------------------------
// CTA-pair form (tile configuration 4): a cluster of two CTAs on two SMs
// computes one 256 x 256 output tile with tcgen05.mma.cta_group::2 (M 256,
// N 256, K 16). CTA r of the pair holds rows [128 r, 128 r + 128) of the A
// tile and rows [128 r, 128 r + 128) of the B tile (three slices each, K
// blocks of 64, two stages) and receives output rows [128 r, 128 r + 128) in
// its own TMEM (2 x 256 columns). The MMA reads each CTA's B half once for
// both SMs, so a CTA's shared memory serves 64 B per clock of operands at the
// full MMA rate instead of the 128 B per clock of the single-CTA 128 x 128
// tile, which is bound by shared-memory bandwidth.
//
// Roles: lane 0 of warp 0 in each CTA loads that CTA's halves, signalling the
// full barrier of CTA 0, whose producer posts the byte count of both; lane 0
// of warp 1 of CTA 0 issues every MMA and commits to the stage-empty and
// accumulator-full barriers of both CTAs at once; the eight epilogue warps of
// each CTA drain their TMEM half and arrive on CTA 0's accumulator-empty
// barrier. Every wait is bounded as in k_gemm_tc_persist.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// shared::cluster address of the same shared variable in CTA `rank`
__device__ __forceinline__ uint32_t map_to_rank(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void tmem_alloc_pair(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
// TMA load into this CTA's shared memory whose completion is counted on an
// mbarrier of either CTA of the pair (bar: shared::cluster address)
__device__ __forceinline__ void tma_load_3d_pair(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                                 uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
      "%4}], [%5];\n" ::"r"(dst),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}
// BF16 x BF16 -> F32, both K-major, M = 256 over the pair, N = 256.
constexpr uint32_t kIdescPair = (1u << 4) | (1u << 7) | (1u << 10) | ((256u >> 3) << 17) | ((256u >> 4) << 24);
__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(da), "l"(db), "r"(kIdescPair), "r"(accumulate), "r"(0)
      : "memory");
}
// commit of this thread's MMAs, arriving on the barrier at the same offset in
// both CTAs of the pair
__device__ __forceinline__ void umma_commit_pair(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n" ::"r"(
          bar),
      "h"((uint16_t)3)
      : "memory");
}

constexpr int kPairBK = 64, kPairS = 2;
constexpr int kPairAB = 128 * kPairBK * 2;                 // one slice of this CTA's A half
constexpr int kPairSB = 6 * kPairAB;                       // three A and three B slice halves
constexpr int kPairSmem = kPairS * kPairSB + kPEpi + 1024 + kPBars;
static_assert(kPairSmem <= 232448, "CTA-pair GEMM shared memory above the per-CTA limit");

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPThreads, 1)
    k_gemm_tc_pair(const TcDesc* __restrict__ descs, const TcWork* __restrict__ work, int nwork,
                   int* __restrict__ status, const unsigned long long* __restrict__ wait_ns) {
  constexpr int S = kPairS, BK = kPairBK, AB = kPairAB, SB = kPairSB;
  constexpr uint32_t TCOLS = 512;  // double-buffered 256-column FP32 accumulator
  static_assert((2 * S + 5) * 8 + 4 <= kPBars, "barrier area");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float* stg_all = reinterpret_cast<float*>(smem + S * SB);
  // full[S] empty[S] accf[2] acce[2] probe, then the TMEM address
  uint64_t* bars = (uint64_t*)(smem + S * SB + kPEpi);
  uint32_t* tmem_slot = (uint32_t*)(smem + S * SB + kPEpi + (2 * S + 5) * 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_rank();
  const bool lead = rank == 0;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[S]);
  const uint32_t accf0 = smem_u32(&bars[2 * S]), acce0 = smem_u32(&bars[2 * S + 2]);
  const uint32_t probe = smem_u32(&bars[2 * S + 4]);
  const uint64_t lim = wait_ns[0];
  if (warp == 0) tmem_alloc_pair(smem_u32(tmem_slot), TCOLS);
  if (tid == 0) {
    for (int b = 0; b < 2 * S + 2; b++) mbar_init(smem_u32(&bars[b]), 1);
    // accumulator-empty: one arrival per epilogue warp of both CTAs (used in CTA 0)
    for (int b = 2 * S + 2; b < 2 * S + 4; b++) mbar_init(smem_u32(&bars[b]), 2 * kPEpiWarps);
    mbar_init(probe, 1);  // probe: nothing ever arrives on it
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  cluster_sync_all();  // both CTAs' barriers initialised before any remote arrival
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int G = gridDim.x >> 1;
  const int cl = blockIdx.x >> 1;
  bool to = false;
  if (wait_ns[1] != 0 && (tid == 0 || tid == 32 || warp >= 2)) {
    if (!mbar_wait(probe, 0, lim)) {
      report_timeout(status, 5, 0);
      to = true;
    }
  }

  if (tid == 0) {  // TMA producer of this CTA's halves
    int g = 0;
    for (int w = cl; w < nwork && !to; w += G) {
      const TcDesc& d = descs[work[w].desc];
      const int tile = work[w].tile;
      const int tm2 = (d.M + 255) / 256;
      const int m0 = (tile % tm2) * 256 + 128 * (int)rank, n0 = (tile / tm2) * 256 + 128 * (int)rank;
      const int nk = d.Kp / BK;
      const int ns = d.nprod == 3 ? 2 : 3;
      for (int kb = 0; kb < nk; kb++, g++) {
        const int s = g % S;
        if (g >= S && !mbar_spin(empty0 + 8 * s, ((g / S) + 1) & 1, lim)) { report_timeout(status, 1, g); to = true; break; }
        const uint32_t fb = map_to_rank(full0 + 8 * s, 0);
        if (lead) mbar_expect_tx(full0 + 8 * s, 2 * ns * 2 * AB);
        const uint32_t st = sbase + s * SB;
        for (int t = 0; t < ns; t++) tma_load_3d_pair(st + t * AB, &d.mapA, kb * BK, m0, t, fb);
        for (int t = 0; t < ns; t++) tma_load_3d_pair(st + (3 + t) * AB, &d.mapB, kb * BK, n0, t, fb);
      }
    }
    // Drain: a stage's loads have landed once the MMAs that read it have
    // completed, which its empty barrier records (in both CTAs).
    for (int gi = g - 1; gi >= 0 && gi >= g - S; gi--)
      if (!mbar_spin(empty0 + 8 * (gi % S), (gi / S) & 1, kDrainLimitNs)) atomicOr(status, 4);
  } else if (tid == 32 && lead) {  // MMA issuer of the pair
    constexpr int pa[6] = {0, 0, 1, 0, 1, 2};
    constexpr int pb[6] = {0, 1, 0, 2, 1, 0};
    const uint64_t d0 = smem_desc_kmajor<BK>(sbase);
    int g = 0, t = 0;
    uint32_t last_bar = 0, last_par = 0;
    for (int w = cl; w < nwork && !to; w += G, t++) {
      const int a = t & 1, u = t >> 1;
      if (t >= 2 && !mbar_spin(acce0 + 8 * a, (u - 1) & 1, lim)) { report_timeout(status, 2, t); to = true; break; }
      tc_fence_after();
      const TcDesc& d = descs[work[w].desc];
      const int nk = d.Kp / BK;
      const int np = d.nprod == 3 ? 3 : 6;
      const uint32_t acc = tmem + a * 256;
      for (int kb = 0; kb < nk; kb++, g++) {
        const int s = g % S;
        if (!mbar_spin(full0 + 8 * s, (g / S) & 1, lim)) { report_timeout(status, 3, g); to = true; break; }
        tc_fence_after();
        const uint64_t ds = d0 + (uint64_t)((uint32_t)(s * SB) >> 4);
#pragma unroll
        for (int p = 0; p < 6; p++) {
          if (p >= np) break;
#pragma unroll
          for (int k16 = 0; k16 < BK / 16; k16++)
            umma_bf16_pair(acc, ds + (uint64_t)((pa[p] * AB + k16 * 32) >> 4),
                           ds + (uint64_t)(((3 + pb[p]) * AB + k16 * 32) >> 4), (kb > 0 || p > 0 || k16 > 0) ? 1u : 0u);
        }
        umma_commit_pair(empty0 + 8 * s);
        last_bar = empty0 + 8 * s;
        last_par = (g / S) & 1;
      }
      if (!to) {
        umma_commit_pair(accf0 + 8 * a);
        last_bar = accf0 + 8 * a;
        last_par = u & 1;
      }
    }
    if (last_bar && !mbar_spin(last_bar, last_par, kDrainLimitNs)) atomicOr(status, 4);
  } else if (warp >= 2) {  // epilogue warps of this CTA's 128 rows
    const int q = warp & 3;
    constexpr int CH = 256 / 64;
    const int c0 = ((warp - 2) >> 2) * CH;
    float* stg = stg_all + (warp - 2) * (32 * 33);
    const uint32_t acce_lead = map_to_rank(acce0, 0);
    int t = 0;
    for (int w = cl; w < nwork && !to; w += G, t++) {
      const int a = t & 1, u = t >> 1;
      if (!mbar_wait(accf0 + 8 * a, u & 1, lim)) { report_timeout(status, 4, t); to = true; break; }
      tc_fence_after();
      const TcDesc& d = descs[work[w].desc];
      const int tile = work[w].tile;
      const int tm2 = (d.M + 255) / 256;
      const int m0 = (tile % tm2) * 256 + 128 * (int)rank, n0 = (tile / tm2) * 256;
      const int r0 = m0 + 32 * q;
      tc_epilogue(d, n0, tmem + a * 256 + ((uint32_t)(32 * q) << 16), r0, lane, stg, c0, c0 + CH);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(acce_lead + 8 * a);
    }
  }
  __syncwarp();
  __syncthreads_or(to);
  tc_fence_before();
  cluster_sync_all();  // both CTAs done with TMEM and with each other's barriers
  tc_fence_after();
  if (warp == 0) tmem_dealloc_pair(tmem, TCOLS);
}

// ---------------------------------------------------------------------------
// FP64 source / residual assembly, split into row-major BF16 slices [i][j]
// through a 32x32 shared-memory transpose.
enum ResKind { RES_NONE = 0, RES_LAP = 1, RES_AOP = 2 };

struct PrepDesc {
  int m, n;
  const double* src;      // v, column-major (m-1)x(n-1)
  double src_scale;       // v = src_scale * src (+ extra)
  const double* bcsrc;    // apply_bc(get_bc(bcsrc, 1.0), 1.0) added to v (vort2flux), or null
  const double* x0;       // residual: v - R(x0), or null
  int res;                // RES_LAP: R = C^T C ; RES_AOP: R = I + nu C^T C
  double nu;
  bf16* Xs;               // 3 slices [i][j], row stride ld, slice stride sX
  long long sX;
  int ld;
};

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// One 32 x 32 tile of one descriptor per block (block map entry {desc, tile},
// tiles numbered i-fastest). The pass is bound by the bytes in flight, so each
// block first issues its whole input at once: each thread's four source values
// as plain loads into registers and, for a residual, x0 with a one-node halo
// (zero outside the grid, which drops the stencil's boundary terms exactly) as
// asynchronous 8-byte copies into shared memory; then it waits once. v is then assembled column-major (a warp reads
// 32 consecutive i) in place and written row-major as three BF16 slices, four
// consecutive j per thread (8-byte stores; a warp writes four 64-byte row
// segments per slice).
__global__ void __launch_bounds__(256, 8) k_prep_split(const PrepDesc* __restrict__ descs,
                                                       const int2* __restrict__ bmap) {
  const int2 bm = bmap[blockIdx.x];
  const PrepDesc& d = descs[bm.x];
  const int M = d.m - 1, N = d.n - 1;
  const int ti = (M + 31) / 32;
  const int i0 = (bm.y % ti) * 32, j0 = (bm.y / ti) * 32;
  __shared__ double t[32][33];
  __shared__ double h[34][35];  // x0(i0 - 1 + a, j0 - 1 + b) at [b][a]
  const double* x0 = d.x0;
  // each thread walks four consecutive rows of one column; its four source
  // values (read by no other thread) go straight to registers, in flight
  // together with the halo copies
  const int tx = threadIdx.x & 31, lb0 = 4 * (threadIdx.x >> 5);
  const int ic = i0 + tx;
  double sv[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int j = j0 + lb0 + r;
    sv[r] = (ic < M && j < N) ? __ldg(d.src + ic + (size_t)j * M) : 0.0;
  }
  if (x0) {
    for (int e = threadIdx.x; e < 34 * 34; e += 256) {
      const int a = e % 34, b = e / 34, i = i0 - 1 + a, j = j0 - 1 + b;
      if (i >= 0 && i < M && j >= 0 && j < N) cp_async8(&h[b][a], x0 + i + (size_t)j * M);
      else h[b][a] = 0.0;
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  // the x0 column values the next row shares stay in registers
  double dn = x0 ? h[lb0][tx + 1] : 0.0, c = x0 ? h[lb0 + 1][tx + 1] : 0.0;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int jj = lb0 + r, j = j0 + jj;
    const double up = x0 ? h[jj + 2][tx + 1] : 0.0;
    t[jj][tx] = 0.0;  // the K padding of the slices reads zero
    if (ic < M && j < N) {
      double v = d.src_scale * sv[r];
      if (d.bcsrc) {
        const int a = ic + 1, b = j + 1;
        if (a == 1 || a == M || b == 1 || b == N)
          v = apply_bc_at(v, a, b, d.m, d.n, 1.0,
                          [&](int side, int I) { return getbc_raw(d.bcsrc, d.m, d.n, side, I) * 1.0; });
      }
      if (x0) {
        // (C^T C x0)(i,j) = 4 x0 - x0(i+-1) - x0(j+-1), zero outside
        double s = 4.0 * c;
        s -= h[jj + 1][tx];
        s -= h[jj + 1][tx + 2];
        s -= dn;
        s -= up;
        const double ax = d.res == RES_LAP ? s : c + d.nu * s;
        v = v - ax;
      }
      t[jj][tx] = v;
    }
    dn = c;
    c = up;
  }
  __syncthreads();
  const int ii = threadIdx.x >> 3, g = threadIdx.x & 7;  // row ii, columns 4g .. 4g+3
  const int i = i0 + ii, j = j0 + 4 * g;
  if (i < M && j < N) {
    bf16 a[4], b[4], c[4];
#pragma unroll
    for (int e = 0; e < 4; e++) split3(t[4 * g + e][ii], a[e], b[e], c[e]);
    bf16* o = d.Xs + (size_t)i * d.ld + j;
    // the row stride and the slice stride are multiples of 64 elements, so
    // every 4-element group starts 8-byte aligned; columns >= N of the last
    // group are zero (the padding the GEMM reads as K)
    store4(o, a);
    store4(o + d.sX, b);
    store4(o + 2 * d.sX, c);
  }
}

// out -= w over a node field (projection, operators.f90:174)
struct AxpyDesc {
  double* out;
  const double* w;
  int count;
};
__global__ void k_sub(const AxpyDesc* __restrict__ ds) {
  const AxpyDesc& d = ds[blockIdx.y];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < d.count; t += gridDim.x * blockDim.x)
    d.out[t] = d.out[t] - d.w[t];
}

// ---------------------------------------------------------------------------
// Host plan
static std::string g_perr;

struct CaseBufs {
  bf16* Xs;    // 3 slices, rows Rm = roundup(m-1,256), ld = Kn = roundup(n-1,64)
  bf16* Ts;    // 3 slices, rows Rn = roundup(n-1,256), ld = Km = roundup(m-1,64)
  long long sX, sT;
  int ldX, ldT;
  const bf16* Sm;  // sine slices for m: rows roundup(m-1,256), ld roundup(m-1,64)
  const bf16* Sn;
  long long sSm, sSn;
  int ldSm, ldSn;
  CUtensorMap mapX, mapT, mapSm, mapSn;      // K blocks of 64: A roles 128 rows, B roles 128 rows
  CUtensorMap mapX2, mapT2, mapSm2, mapSn2;  // K blocks of 32: A roles 128 rows, B roles 256 rows
  CUtensorMap mapT3, mapSn3;                 // K blocks of 32: B roles 128 rows
  const float* lamx;
  const float* lamy;
};

struct PrecisionPlan {
  std::vector<CaseBufs> bufs;  // indexed like the case array of the handle
  std::map<int, std::pair<bf16*, long long>> sine;  // N+1 -> slices
  std::map<int, float*> lam;                        // N+1 -> 1-D eigenvalues
  int* status = nullptr;
  unsigned long long* wait_ns = nullptr;  // device words: limit of the GEMM's waits (ns), probe flag
  int tc_tile = 0;                        // tile configuration: 0 = the measured autotuner, 1..4
  int refine_slices = 0;                  // slices per operand of the correction solves: 0 = by kind, 2 or 3
  int poisson_sweeps = 1;                 // correction sweeps of the Poisson (ctci) solves: 1 or 2
  std::vector<int> tile_choice;           // configuration of each GEMM launch group, in build order
  Alloc alloc;
};

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static int g_num_sms = 0;
static int g_pair_clusters = 0;  // CTA pairs of k_gemm_tc_pair resident at once (0: configuration 4 unavailable)

static inline int rup(int x, int a) { return (x + a - 1) / a * a; }

// 3-D map over [slice][row][k] BF16 (k contiguous): box bk x box_rows x 1,
// swizzle matching the row length (bk=64: 128 B, bk=32: 64 B).
static bool make_map(CUtensorMap* map, const bf16* base, int ld, int rows, long long slice_stride, int bk,
                     int box_rows) {
  cuuint64_t dims[3] = {(cuuint64_t)ld, (cuuint64_t)rows, 3};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)slice_stride * 2};
  cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void*)base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}



// lambda(i) = 2 - 2 cos(pi (i+1) / m) = 4 sin^2(pi (i+1) / 2m), free of cancellation.
static float* lam_table(PrecisionPlan* pp, int m) {
  auto it = pp->lam.find(m);
  if (it != pp->lam.end()) return it->second;
  std::vector<float> h(m - 1);
  for (int i = 0; i < m - 1; i++) {
    double sn = std::sin(M_PI * (double)(i + 1) / (2.0 * m));
    h[i] = (float)(4.0 * sn * sn);
  }
  float* d = (float*)pp->alloc(sizeof(float) * h.size());
  if (d) cudaMemcpy(d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
  pp->lam[m] = d;
  return d;
}


static std::pair<bf16*, long long> sine_slices(PrecisionPlan* pp, int m) {
  auto it = pp->sine.find(m);
  if (it != pp->sine.end()) return it->second;
  int N = m - 1, R = rup(N, 256), ld = rup(N, 64);  // rows serve both GEMM roles
  long long sl = (long long)R * ld;
  std::vector<uint16_t> h((size_t)3 * sl, 0);
  for (int a = 0; a < N; a++)
    for (int b = 0; b < N; b++) {
      long long p = ((long long)(a + 1) * (b + 1)) % (2 * m);
      double x = 2.0 * std::sin(M_PI * (double)p / (double)m);
      // round-to-nearest-even splits of x into three bf16 values
      double r = x;
      for (int s = 0; s < 3; s++) {
        float f = (float)r;
        uint32_t u;
        memcpy(&u, &f, 4);
        uint32_t lsb = (u >> 16) & 1u;
        u += 0x7FFFu + lsb;
        uint16_t hb = (uint16_t)(u >> 16);
        h[(size_t)s * sl + (size_t)a * ld + b] = hb;
        uint32_t back = (uint32_t)hb << 16;
        float fb;
        memcpy(&fb, &back, 4);
        r = r - (double)fb;
      }
    }
  bf16* d = (bf16*)pp->alloc(h.size() * 2);
  if (d) cudaMemcpy(d, h.data(), h.size() * 2, cudaMemcpyHostToDevice);
  pp->sine[m] = {d, sl};
  return pp->sine[m];
}

int precision_init(PrecisionPlan*& pp, cudaStream_t, const std::vector<DevCase>& cases, const DevCase*,
                   Alloc alloc) {
  pp = new PrecisionPlan();
  pp->alloc = alloc;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_gemm_tc_persist<128, 64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tc_smem<128, 64, 2>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_gemm_tc_persist<256, 32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tc_smem<256, 32, 2>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_gemm_tc_persist<128, 32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tc_smem<128, 32, 4>()) != cudaSuccess ||
        cudaFuncSetAttribute(k_gemm_tc_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairSmem) != cudaSuccess) {
      g_perr = "cannot raise shared memory limit for the tensor-core GEMM";
      return 4;
    }
    attr = true;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeClusterDimension;
    la[0].val.clusterDim.x = 2;
    la[0].val.clusterDim.y = 1;
    la[0].val.clusterDim.z = 1;
    lc.gridDim = dim3(2 * std::max(1, g_num_sms / 2));
    lc.blockDim = dim3(kPThreads);
    lc.dynamicSmemBytes = kPairSmem;
    lc.attrs = la;
    lc.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, k_gemm_tc_pair, &lc) != cudaSuccess) {
      cudaGetLastError();
      nc = 0;
    }
    g_pair_clusters = nc;
  }
  pp->status = cases.empty() ? (int*)alloc(sizeof(int) * 4) : cases[0].status;
  pp->wait_ns = (unsigned long long*)alloc(2 * sizeof(unsigned long long));
  if (!pp->wait_ns) {
    g_perr = "device allocation failed for the wait limit";
    return 8;
  }
  if (precision_set_wait_limit(pp, (double)kWaitLimitNs * 1e-9, 0)) {
    g_perr = "cannot set the wait limit";
    return 4;
  }
  if (!g_encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn) {
      g_perr = "cuTensorMapEncodeTiled is not available";
      return 4;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  for (auto& c : cases) {
    CaseBufs b{};
    // rows of X and T padded to the widest tile (256)
    int Rm = rup(c.m - 1, 256), Rn = rup(c.n - 1, 256), Km = rup(c.m - 1, 64), Kn = rup(c.n - 1, 64);
    b.sX = (long long)Rm * Kn;
    b.sT = (long long)Rn * Km;
    b.ldX = Kn;
    b.ldT = Km;
    b.Xs = (bf16*)alloc(sizeof(bf16) * 3 * b.sX);
    b.Ts = (bf16*)alloc(sizeof(bf16) * 3 * b.sT);
    auto sm = sine_slices(pp, c.m);
    auto sn = sine_slices(pp, c.n);
    b.Sm = sm.first; b.sSm = sm.second; b.ldSm = Km;
    b.Sn = sn.first; b.sSn = sn.second; b.ldSn = Kn;
    b.lamx = lam_table(pp, c.m);
    b.lamy = lam_table(pp, c.n);
    if (!b.Xs || !b.Ts || !b.Sm || !b.Sn || !pp->status || !b.lamx || !b.lamy) {
      g_perr = "device allocation failed for the split-precision buffers";
      return 8;
    }
    const int Rs_m = rup(c.m - 1, 256), Rs_n = rup(c.n - 1, 256);
    if (!make_map(&b.mapX, b.Xs, Kn, Rm, b.sX, 64, 128) || !make_map(&b.mapT, b.Ts, Km, Rn, b.sT, 64, 128) ||
        !make_map(&b.mapSm, b.Sm, Km, Rs_m, b.sSm, 64, 128) || !make_map(&b.mapSn, b.Sn, Kn, Rs_n, b.sSn, 64, 128) ||
        !make_map(&b.mapX2, b.Xs, Kn, Rm, b.sX, 32, 128) || !make_map(&b.mapT2, b.Ts, Km, Rn, b.sT, 32, 256) ||
        !make_map(&b.mapSm2, b.Sm, Km, Rs_m, b.sSm, 32, 128) ||
        !make_map(&b.mapSn2, b.Sn, Kn, Rs_n, b.sSn, 32, 256) || !make_map(&b.mapT3, b.Ts, Km, Rn, b.sT, 32, 128) ||
        !make_map(&b.mapSn3, b.Sn, Kn, Rs_n, b.sSn, 32, 128)) {
      g_perr = "cuTensorMapEncodeTiled failed";
      return 4;
    }
    pp->bufs.push_back(b);
  }
  return 0;
}

void precision_free(PrecisionPlan* pp) { delete pp; }

void precision_set_tile(PrecisionPlan* pp, int cfg) { pp->tc_tile = (cfg >= 1 && cfg <= kTcCfgs) ? cfg : 0; }
void precision_set_refine(PrecisionPlan* pp, int slices, int poisson_sweeps) {
  pp->refine_slices = (slices == 2 || slices == 3) ? slices : 0;
  pp->poisson_sweeps = poisson_sweeps == 2 ? 2 : 1;
}
const std::vector<int>& precision_tile_choices(const PrecisionPlan* pp) { return pp->tile_choice; }
void precision_reset_tile_choices(PrecisionPlan* pp) { pp->tile_choice.clear(); }

int precision_set_wait_limit(PrecisionPlan* pp, double seconds, int probe) {
  if (!pp || !pp->wait_ns || !(seconds >= 0.0) || seconds > 60.0) return 7;
  const unsigned long long w[2] = {(unsigned long long)(seconds * 1e9), probe ? 1ull : 0ull};
  return cudaMemcpy(pp->wait_ns, w, sizeof(w), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : 4;
}
const char* precision_error() { return g_perr.c_str(); }

// One solve request: x = A^-1 v for one (case, level) item.
struct SolveReq {
  int c;              // index into pp->bufs
  const DevCase* hc;  // host copy of the case
  int k;              // level (1-based), for del22
  int fkind;          // F_LAMINV (ctci) or F_LAM1I_NORM (A = I + nu C^T C)
  PrepDesc src;       // how to assemble v (Xs and ld filled in here)
  double* out;        // x (column-major FP64)
  bool presplit;      // v's slices are already in the case's X buffer: pass 0 needs no assembly
};

template <class T>
static T* upload(PrecisionPlan* pp, const std::vector<T>& v) {
  T* p = (T*)pp->alloc(sizeof(T) * std::max<size_t>(1, v.size()));
  if (p && !v.empty()) cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
  return p;
}

// Output tile of a tile configuration (1..4, see kTcCfgs above).
static inline int tc_bn(int cfg) { return cfg == 2 || cfg == 4 ? 256 : 128; }
static inline int tc_bm(int cfg) { return cfg == 4 ? 256 : 128; }

// Work list of one launch group for tile configuration cfg: every tile of
// every descriptor, sorted by K length (longest first) for balance across the
// SMs (across the CTA pairs for configuration 4).
static std::vector<TcWork> tc_work(const std::vector<TcDesc>& ds, int cfg) {
  const int bn = tc_bn(cfg), bm = tc_bm(cfg);
  std::vector<TcWork> wl;
  for (int i = 0; i < (int)ds.size(); i++) {
    const int tiles = ((ds[i].M + bm - 1) / bm) * ((ds[i].N + bn - 1) / bn);
    for (int t = 0; t < tiles; t++) wl.push_back({i, t});
  }
  std::stable_sort(wl.begin(), wl.end(), [&](const TcWork& x, const TcWork& y) { return ds[x.desc].Kp > ds[y.desc].Kp; });
  return wl;
}

static void launch_tc(int cfg, const TcDesc* dd, const TcWork* dw, int nw, int* status,
                      const unsigned long long* wait_ns, cudaStream_t st) {
  if (cfg == 4) {
    // one CTA pair per two SMs, at most as many pairs as fit at once
    const int pairs = std::max(1, std::min(nw, g_pair_clusters));
    k_gemm_tc_pair<<<2 * pairs, kPThreads, kPairSmem, st>>>(dd, dw, nw, status, wait_ns);
    return;
  }
  const int grid = std::min(nw, g_num_sms > 0 ? g_num_sms : 148);
  if (cfg == 2)
    k_gemm_tc_persist<256, 32, 2><<<grid, kPThreads, tc_smem<256, 32, 2>(), st>>>(dd, dw, nw, status, wait_ns);
  else if (cfg == 3)
    k_gemm_tc_persist<128, 32, 4><<<grid, kPThreads, tc_smem<128, 32, 4>(), st>>>(dd, dw, nw, status, wait_ns);
  else
    k_gemm_tc_persist<128, 64, 2><<<grid, kPThreads, tc_smem<128, 64, 2>(), st>>>(dd, dw, nw, status, wait_ns);
}

// Measured autotuner of the tensor-core GEMM's tile configuration. A launch
// group is timed once with each configuration -- its outputs redirected to a
// scratch buffer, its operands read where they lie, so no state changes --
// and the fastest is kept, cached per process and device by the group's shape
// signature. All configurations issue the same slice products; only the order
// of the FP32 accumulation differs (K blocks of 32 against 64), which the
// refinement's FP64 residual absorbs.
static std::mutex g_tc_mu;
static std::map<std::string, int> g_tc_tuned;

static std::string tc_signature(const std::vector<TcDesc>& ds) {
  std::vector<std::string> parts;
  for (auto& d : ds)
    parts.push_back(std::to_string(d.M) + "x" + std::to_string(d.N) + "x" + std::to_string(d.Kp) + ":" +
                    std::to_string(d.epi) + "/" + std::to_string(d.nprod));
  std::sort(parts.begin(), parts.end());
  int dev = 0;
  cudaGetDevice(&dev);
  std::string key = "dev" + std::to_string(dev) + "|";
  for (auto& p : parts) key += p + ";";
  return key;
}

static int tune_tc(PrecisionPlan* pp, const std::vector<TcDesc>& ds, cudaStream_t st) {
  const std::string key = tc_signature(ds);
  std::lock_guard<std::mutex> lk(g_tc_mu);
  auto it = g_tc_tuned.find(key);
  if (it != g_tc_tuned.end()) return it->second;
  size_t need = 16;
  for (auto& d : ds) {
    if (d.epi == TC_SPLIT_COL || d.epi == TC_SCALE_SPLIT_ROW) need = std::max(need, (size_t)(3 * d.sC) * sizeof(bf16));
    else need = std::max(need, (size_t)d.ldc * d.N * sizeof(double));
  }
  int best = 1;
  void* scratch = nullptr;
  TcDesc* dd = nullptr;
  TcWork* dw = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<TcDesc> t = ds;
  size_t maxw = 0;
  for (int cfg = 1; cfg <= kTcCfgs; cfg++) maxw = std::max(maxw, tc_work(ds, cfg).size());
  if (cudaMalloc(&scratch, need) == cudaSuccess && cudaMalloc(&dd, sizeof(TcDesc) * t.size()) == cudaSuccess &&
      cudaMalloc(&dw, sizeof(TcWork) * maxw) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
      cudaEventCreate(&e1) == cudaSuccess) {
    cudaMemsetAsync(scratch, 0, need, st);
    for (auto& d : t) {
      if (d.Cs) d.Cs = (bf16*)scratch;
      if (d.C64) d.C64 = (double*)scratch;
    }
    cudaMemcpy(dd, t.data(), sizeof(TcDesc) * t.size(), cudaMemcpyHostToDevice);
    float best_ms = 1e30f;
    for (int cfg = 1; cfg <= kTcCfgs; cfg++) {
      if (cfg == 4 && g_pair_clusters == 0) continue;
      const std::vector<TcWork> wl = tc_work(ds, cfg);
      cudaMemcpy(dw, wl.data(), sizeof(TcWork) * wl.size(), cudaMemcpyHostToDevice);
      const int nw = (int)wl.size();
      launch_tc(cfg, dd, dw, nw, pp->status, pp->wait_ns, st);  // warm-up
      if (cudaGetLastError() != cudaSuccess) continue;  // a configuration that cannot launch here is not timed
      cudaEventRecord(e0, st);
      for (int r = 0; r < 3; r++) launch_tc(cfg, dd, dw, nw, pp->status, pp->wait_ns, st);
      cudaEventRecord(e1, st);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess &&
          ms < best_ms) {
        best_ms = ms;
        best = cfg;
      }
    }
  }
  cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (dw) cudaFree(dw);
  if (dd) cudaFree(dd);
  if (scratch) cudaFree(scratch);
  g_tc_tuned[key] = best;
  return best;
}

// One persistent launch over every tile of every descriptor, with the tile
// configuration the handle's option or the autotuner chose.
static void add_gemm_persist(PrecisionPlan* pp, Prog& P, const std::vector<TcDesc>& ds, cudaStream_t st) {
  if (ds.empty()) return;
  int cfg = pp->tc_tile >= 1 && pp->tc_tile <= kTcCfgs ? pp->tc_tile : tune_tc(pp, ds, st);
  if (cfg == 4 && g_pair_clusters == 0) cfg = 1;  // no CTA pair fits on this device
  pp->tile_choice.push_back(cfg);
  std::vector<TcWork> wl = tc_work(ds, cfg);
  double fl = 0.0;
  for (auto& d : ds) fl += 2.0 * d.M * (double)d.N * (double)(d.epi == TC_SPLIT_COL ? d.N : d.M);
  TcDesc* dd = upload(pp, ds);
  TcWork* dw = upload(pp, wl);
  const int nw = (int)wl.size();
  int* status = pp->status;
  const unsigned long long* wait_ns = pp->wait_ns;
  P.push_back({[=]() { launch_tc(cfg, dd, dw, nw, status, wait_ns, st); }, TAG_GEMM_TC, fl});
}

static void add_gemm(PrecisionPlan* pp, Prog& P, const std::vector<TcDesc>& all, cudaStream_t st) {
  add_gemm_persist(pp, P, all, st);
}

static void add_prep(PrecisionPlan* pp, Prog& P, const std::vector<PrepDesc>& ds, cudaStream_t st) {
  if (ds.empty()) return;
  std::vector<int2> map;
  for (int i = 0; i < (int)ds.size(); i++) {
    int tiles = ((ds[i].m - 1 + 31) / 32) * ((ds[i].n - 1 + 31) / 32);
    for (int t = 0; t < tiles; t++) map.push_back(make_int2(i, t));
  }
  PrepDesc* dd = upload(pp, ds);
  const int2* dm = upload(pp, map);
  const int nb = (int)map.size();
  P.push_back({[=]() { k_prep_split<<<nb, 256, 0, st>>>(dd, dm); }, TAG_SPLIT, 0.0});
}

// The eight GEMMs + two assembly passes of a batch of refined solves.
// Refinement of a batch of solves of one kind. Each correction pass forms the
// residual r = v - A x in FP64 with the exact 5-point stencil and adds S f S r.
// Why the Poisson solves (ctci, A = C^T C) may need a second correction sweep
// (poisson_sweeps = 2; one is the default): the
// FP32 accumulation leaves white noise of relative size e ~ 3e-7 in x; A
// lifts its high modes (lambda up to 8) into r, and the noise of the next
// transform of r, spread back over all modes, is lifted by 1/lambda_min at the
// low modes, so each sweep contracts the error only by kappa*e, kappa =
// lambda_max/lambda_min ~ 0.4 m^2 (~0.03 at m = 512). The Crank-Nicolson and
// ainv operators, A = I + nu C^T C, have kappa = 1 + 8 nu (~1-5): one sweep
// with two slices per operand (three products) leaves ~1e-11 there.
static void build_solves(PrecisionPlan* pp, Prog& P, std::vector<SolveReq>& rq, cudaStream_t st) {
  if (rq.empty()) return;
  const bool poisson = rq[0].fkind == F_LAMINV;
  const int npass = 1 + (poisson ? pp->poisson_sweeps : 1);
  // slice products of a correction pass: three slices (six products) for the
  // Poisson solves, two (three products) for the others, unless fixed
  const int np_corr = pp->refine_slices == 3 ? 6 : pp->refine_slices == 2 ? 3 : (poisson ? 6 : 3);
  for (int pass = 0; pass < npass; pass++) {
    std::vector<PrepDesc> prep;
    std::vector<TcDesc> g1, g2, g3, g4;
    for (auto& r : rq) {
      const CaseBufs& b = pp->bufs[r.c];
      const DevCase& c = *r.hc;
      PrepDesc pd = r.src;
      pd.m = c.m; pd.n = c.n;
      pd.Xs = b.Xs; pd.sX = b.sX; pd.ld = b.ldX;
      if (pass >= 1) {
        pd.x0 = r.out;
        pd.res = r.fkind == F_LAMINV ? RES_LAP : RES_AOP;
        pd.nu = 0.5 * c.dt / (c.delta * c.delta * std::pow(4.0, r.k - 1) * c.re);
      } else {
        pd.x0 = nullptr;
      }
      if (!(pass == 0 && r.presplit)) prep.push_back(pd);
      int M = c.m - 1, N = c.n - 1;
      int tm = (M + 127) / 128;
      TcDesc R{};  // T = X * S_n
      R.mapA = b.mapX; R.mapB = b.mapSn;
      R.mapA2 = b.mapX2; R.mapB2 = b.mapSn2; R.mapB3 = b.mapSn3;
      R.M = M; R.N = N; R.Kp = rup(N, 64); R.tiles_m = tm;
      R.epi = TC_SPLIT_COL; R.Cs = b.Ts; R.sC = b.sT; R.ldcs = b.ldT;
      TcDesc L1{};  // U = f .* (S_m * T)
      L1.mapA = b.mapSm; L1.mapB = b.mapT;
      L1.mapA2 = b.mapSm2; L1.mapB2 = b.mapT2; L1.mapB3 = b.mapT3;
      L1.M = M; L1.N = N; L1.Kp = rup(M, 64); L1.tiles_m = tm;
      L1.epi = TC_SCALE_SPLIT_ROW; L1.fkind = r.fkind; L1.Cs = b.Xs; L1.sC = b.sX; L1.ldcs = b.ldX;
      L1.lamx = b.lamx; L1.lamy = b.lamy; L1.norm = (float)c.norm;
      L1.nu = (float)(0.5 * c.dt / (c.delta * c.delta * std::pow(4.0, r.k - 1) * c.re));
      TcDesc L2 = L1;  // x = S_m * T'
      L2.epi = pass == 0 ? TC_F64_STORE : TC_F64_ADD;
      L2.C64 = r.out; L2.ldc = M;
      const int np = pass == 0 ? 6 : np_corr;
      R.nprod = np;
      L1.nprod = np;
      L2.nprod = np;
      g1.push_back(R);
      g2.push_back(L1);
      g3.push_back(R);
      g4.push_back(L2);
    }
    add_prep(pp, P, prep, st);
    add_gemm(pp, P, g1, st);
    add_gemm(pp, P, g2, st);
    add_gemm(pp, P, g3, st);
    add_gemm(pp, P, g4, st);
  }
}

void build_precision_step1(PrecisionPlan* pp, Prog& P, const DevCase* dcases, const std::vector<DevCase>& cs,
                           cudaStream_t st) {
  int Lmax = 0, mns = 0;
  for (auto& c : cs) { Lmax = std::max(Lmax, c.L); mns = std::max(mns, c.ns); }
  for (int t = 0; t < Lmax; t++) {
    std::vector<LevelItem> it;
    std::vector<int> cnt;
    std::vector<SolveReq> rq;
    for (size_t i = 0; i < cs.size(); i++) {
      const DevCase& c = cs[i];
      int k = c.L - t;
      if (k < 1) continue;
      it.push_back({(int)i, k});
      cnt.push_back(c.ns);
      // b = norm*rhsA + (I - nu_k C^T C) omega_k ; omega_k <- A_k^-1 b
      SolveReq r{};
      r.c = (int)i; r.hc = &cs[i]; r.k = k; r.fkind = F_LAM1I_NORM;
      r.out = c.omega + (size_t)(k - 1) * c.ns;
      // the correction residual's right-hand side is b itself (wd)
      r.src.src = c.wd; r.src.src_scale = 1.0;
      r.presplit = true;
      rq.push_back(r);
    }
    // b = norm*rhsA + (I - nu_k C^T C) omega_k is assembled once, in the same
    // pass as the nonlinear term (k_rhs_split): FP64 copy in wd for the
    // correction residual, BF16 slices for the first solve; b must be formed
    // before omega_k is overwritten by x0
    std::vector<RhsSplitDesc> sd;
    std::vector<int2> tmap;
    for (size_t q = 0; q < rq.size(); q++) {
      SolveReq& r = rq[q];
      const DevCase& c = *r.hc;
      const CaseBufs& b = pp->bufs[r.c];
      const double nu = 0.5 * c.dt / (c.delta * c.delta * std::pow(4.0, r.k - 1) * c.re);
      sd.push_back({c.norm, nu, c.wd, reinterpret_cast<uint16_t*>(b.Xs), b.sX, b.ldX});
      const int tiles = ((c.m - 1 + 31) / 32) * ((c.n - 1 + 31) / 32);
      for (int t = 0; t < tiles; t++) tmap.push_back(make_int2((int)q, t));
    }
    LevelItem* d_it = upload(pp, it);
    const RhsSplitDesc* d_sd = upload(pp, sd);
    const int2* d_tm = upload(pp, tmap);
    const int ntm = (int)tmap.size();
    P.push_back({[=]() { launch_rhs_split(dcases, d_it, d_sd, d_tm, ntm, 0, st); }, TAG_STENCIL, 0.0});
    build_solves(pp, P, rq, st);
  }
}

void build_precision_vort2flux(PrecisionPlan* pp, Prog& P, const DevCase* dcases, const std::vector<DevCase>& cs,
                               const std::vector<int>& ids, bool curl_all, cudaStream_t st) {
  int Lmax = 0, mns = 0, mnq = 0;
  for (auto& c : cs) { Lmax = std::max(Lmax, c.L); mns = std::max(mns, c.ns); mnq = std::max(mnq, c.nq); }
  for (int k = 2; k <= Lmax; k++) {
    std::vector<LevelItem> it;
    std::vector<int> cnt;
    for (size_t i = 0; i < cs.size(); i++)
      if (cs[i].L >= k) { it.push_back({ids[i], k}); cnt.push_back(coarsify_count(cs[i].m, cs[i].n)); }
    if (it.empty()) continue;
    LevelItem* d = upload(pp, it);
    const std::vector<int2> bmv = block_map(cnt);
    const int2* bm = upload(pp, bmv);
    const int nbm = (int)bmv.size();
    P.push_back({[=]() { launch_coarsify(dcases, d, bm, nbm, st); }, TAG_STENCIL, 0.0});
  }
  for (int t = 0; t < Lmax; t++) {
    std::vector<SolveReq> rq;
    for (size_t i = 0; i < cs.size(); i++) {
      const DevCase& c = cs[i];
      int k = c.L - t;
      if (k < 1) continue;
      SolveReq r{};
      r.c = (int)i; r.hc = &cs[i]; r.k = k; r.fkind = F_LAMINV;
      r.src.src = c.omega + (size_t)(k - 1) * c.ns; r.src.src_scale = 1.0;
      r.src.bcsrc = k < c.L ? c.s + (size_t)k * c.ns : nullptr;
      r.out = c.s + (size_t)(k - 1) * c.ns;
      rq.push_back(r);
    }
    build_solves(pp, P, rq, st);
  }
  std::vector<LevelItem> ci;
  std::vector<int> cnt;
  for (size_t i = 0; i < cs.size(); i++)
    for (int k = 1; k <= (curl_all ? cs[i].L : 1); k++) { ci.push_back({ids[i], k}); cnt.push_back(cs[i].nq); }
  LevelItem* d = upload(pp, ci);
  const std::vector<int2> bmv = block_map(cnt);
  const int2* bm = upload(pp, bmv);
  const int nbm = (int)bmv.size();
  P.push_back({[=]() { launch_curl(dcases, d, bm, nbm, st); }, TAG_STENCIL, 0.0});
}

void build_precision_ainv(PrecisionPlan* pp, Prog& P, const DevCase* dcases, const std::vector<DevCase>& cs,
                          int final_epi, cudaStream_t st) {
  (void)dcases;
  std::vector<SolveReq> rq;
  std::vector<AxpyDesc> ax;
  for (size_t i = 0; i < cs.size(); i++) {
    const DevCase& c = cs[i];
    SolveReq r{};
    r.c = (int)i; r.hc = &cs[i]; r.k = 1; r.fkind = F_LAM1I_NORM;
    r.src.src = c.vort; r.src.src_scale = 1.0;
    r.out = final_epi == EPI_SUBTRACT ? c.wd : c.omega;
    rq.push_back(r);
    ax.push_back({c.omega, c.wd, c.ns});
  }
  build_solves(pp, P, rq, st);
  if (final_epi == EPI_SUBTRACT) {
    AxpyDesc* d = upload(pp, ax);
    int n = (int)ax.size(), mns = 0;
    for (auto& c : cs) mns = std::max(mns, c.ns);
    P.push_back({[=]() {
                   dim3 g((mns + 255) / 256, n);
                   k_sub<<<g, 256, 0, st>>>(d);
                 },
                 TAG_STENCIL, 0.0});
  }
}

int precision_apply_op(PrecisionPlan* pp, int op, const DevCase* ds, const DevCase& s, cudaStream_t st) {
  (void)ds;
  // op 1 (ctci) and op 2 (ainv) as refined split-precision solves of case 0's buffers
  if (op != 1 && op != 2) return 7;
  Prog P;
  std::vector<DevCase> one{s};
  std::vector<SolveReq> rq(1);
  rq[0].c = 0; rq[0].hc = &one[0]; rq[0].k = 1;
  rq[0].fkind = op == 1 ? F_LAMINV : F_LAM1I_NORM;
  rq[0].src.src = s.vort; rq[0].src.src_scale = op == 1 ? 1.0 : 1.0;
  rq[0].out = s.omega;
  const size_t nchoice = pp->tile_choice.size();
  build_solves(pp, P, rq, st);
  pp->tile_choice.resize(nchoice);  // the step program's record stays as it was
  for (auto& e : P) e.fn();
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return 4;
  int st4[4] = {0, 0, 0, 0};
  cudaMemcpy(st4, pp->status, sizeof(st4), cudaMemcpyDeviceToHost);
  if (!st4[0]) return 0;
  cudaMemset(pp->status, 0, sizeof(st4));
  g_perr = "tensor-core GEMM: a bounded wait gave up (role " + std::to_string(st4[1]) + ", block " +
           std::to_string(st4[2]) + ", step " + std::to_string(st4[3]) + ")";
  return 6;
}

}  // namespace ibfs
