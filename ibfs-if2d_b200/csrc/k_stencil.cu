// k_stencil.cu -- HBM-bound stencil, inter-level and immersed-boundary kernels
// of the IBFS advance. Each kernel follows the reference loop it replaces
// (atchieu/ibfs-if2d src/operators.f90, cited per kernel); all arithmetic is
// FP64. Grids are grouped: blockIdx.y selects a (case, level) item.
#include <cuda_bf16.h>

#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"

namespace ibfs {

// ---------------------------------------------------------------------------
// lastbc(:,k) = get_bc(omega(:,:,k+1), 0.25) for k<L; lastbc(:,L) = 0
// (operators.f90:97-100). One thread per ring entry.
__global__ void k_lastbc(const DevCase* __restrict__ cases, const LevelItem* __restrict__ items) {
  LevelItem it = items[blockIdx.y];
  const DevCase& C = cases[it.c];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C.nring) return;
  int m = C.m, n = C.n;
  double* ring = C.lastbc + (size_t)(it.k - 1) * C.nring;
  if (it.k >= C.L) {
    ring[t] = 0.0;
    return;
  }
  int side, I;
  if (t < n + 1) { side = SIDE_LEFT; I = t + 1; }
  else if (t < 2 * (n + 1)) { side = SIDE_RIGHT; I = t - (n + 1) + 1; }
  else if (t < 2 * (n + 1) + m + 1) { side = SIDE_BOTTOM; I = t - 2 * (n + 1) + 1; }
  else { side = SIDE_TOP; I = t - 2 * (n + 1) - (m + 1) + 1; }
  const double* r = C.omega + (size_t)it.k * C.ns;  // level k+1
  ring[t] = getbc_raw(r, m, n, side, I) * 0.25;
}

// ---------------------------------------------------------------------------
// Fused rhs of the per-level vorticity update (operators.f90:104-133):
//   rhs    = rot(nonlinear(omega_k, q_k, q0_k, lastbc_k))       (:112, :465-510, :291-304)
//   [first step] rhs_old = rhs                                   (:115-117)
//   rhsbc  = apply_bc(lastbc_k)*vfac + apply_bc(omega_bc)*vfac   (:121-123)
//   rhsA   = con1*rhs + con2*rhs_old + rhsbc                     (:127-129)
//   rhs_old= rhs                                                 (:133)
// omega_bc = get_bc(omega_{k+1}^new, 0.25) is gathered on the fly.
__device__ __forceinline__ double vavg_at(const double* __restrict__ q, const double* __restrict__ q0, int i, int j,
                                          int m, int n) {
  int a = voff(i, j, m, n), b = voff(i - 1, j, m, n);
  return 0.5 * (q[a] + q[b] + q0[a] + q0[b]);
}
__device__ __forceinline__ double uavg_at(const double* __restrict__ q, const double* __restrict__ q0, int i, int j,
                                          int m) {
  int a = uoff(i, j, m), b = uoff(i, j - 1, m);
  return 0.5 * (q[a] + q[b] + q0[a] + q0[b]);
}
// The same averages with q0 in closed form (u-faces u0, v-faces 0): the
// reference's sums with the q0 terms in place, so the values are identical.
__device__ __forceinline__ double vavg_c(const double* __restrict__ q, int i, int j, int m, int n) {
  int a = voff(i, j, m, n), b = voff(i - 1, j, m, n);
  return 0.5 * (q[a] + q[b] + 0.0 + 0.0);
}
__device__ __forceinline__ double uavg_c(const double* __restrict__ q, double u0, int i, int j, int m) {
  int a = uoff(i, j, m), b = uoff(i, j - 1, m);
  return 0.5 * (q[a] + q[b] + u0 + u0);
}

// The per-node values of the level update's right-hand side: returns rhsA =
// con1*rhs + con2*rhs_old + rhsbc and stores rhs_old = rhs (operators.f90:112-133).
template <bool Q0C>
__device__ __forceinline__ double rhs_value(const DevCase& C, LevelItem it, int t, int first_step) {
  int m = C.m, n = C.n;
  int i = t % (m - 1) + 2, j = t / (m - 1) + 2;
  int k = it.k;
  const double* om = C.omega + (size_t)(k - 1) * C.ns;
  const double* q = C.q + (size_t)(k - 1) * C.nq;
  const double* q0 = C.q0 + (size_t)(k - 1) * C.nq;
  const double u0 = C.q0_u1 * (double)(1 << (k - 1));
  const double* bc = C.lastbc + (size_t)(k - 1) * C.nring;
  int bottom = 2 * (n + 1), top = 2 * (n + 1) + m + 1, right = n + 1;
  // omega extended with the ring along j (column i) and along i (row j)
  auto Wj = [&](int jj) -> double {
    if (jj == 1) return bc[bottom + i - 1];
    if (jj == n + 1) return bc[top + i - 1];
    return om[nidx(i, jj, m)];
  };
  auto Wi = [&](int ii, int jj) -> double {
    if (ii == 1) return bc[jj - 1];
    if (ii == m + 1) return bc[right + jj - 1];
    return om[nidx(ii, jj, m)];
  };
  auto vavg = [&](int ii, int jj) -> double { return Q0C ? vavg_c(q, ii, jj, m, n) : vavg_at(q, q0, ii, jj, m, n); };
  auto uavg = [&](int ii, int jj) -> double { return Q0C ? uavg_c(q, u0, ii, jj, m) : uavg_at(q, q0, ii, jj, m); };
  auto fqu = [&](int jj) -> double {  // fq(u(i,jj)), jj = 1..n
    return 0.5 * (vavg(i, jj + 1) * Wj(jj + 1) + vavg(i, jj) * Wj(jj));
  };
  auto fqv = [&](int ii) -> double {  // fq(v(ii,j)), ii = 1..m
    return -0.5 * (uavg(ii + 1, j) * Wi(ii + 1, j) + uavg(ii, j) * Wi(ii, j));
  };
  double rhs = fqv(i) - fqv(i - 1) - fqu(j) + fqu(j - 1);

  double* ro = C.rhs_old + (size_t)(k - 1) * C.ns;
  // explicit Euler on the first step (itime == 1), operators.f90:115-117
  double rold = (first_step || *C.itime == 1) ? rhs : ro[t];
  // rhsbc: two apply_bc passes onto zero, each in the reference's order
  double vf = 0.5 * C.dt / C.re / (C.delta * C.delta * (double)(1 << (2 * (k - 1)))) / C.norm;
  int a = i - 1, b = j - 1;
  double rb = 0.0;
  if (a == 1 || a == m - 1 || b == 1 || b == n - 1) {
    rb = apply_bc_at(rb, a, b, m, n, vf, [&](int side, int I) { return ring_at(bc, m, n, side, I); });
    if (k < C.L) {
      const double* cr = C.omega + (size_t)k * C.ns;  // omega_{k+1}, already advanced
      rb = apply_bc_at(rb, a, b, m, n, vf,
                       [&](int side, int I) { return getbc_raw(cr, m, n, side, I) * 0.25; });
    } else {
      rb = apply_bc_at(rb, a, b, m, n, vf, [&](int, int) { return 0.0; });
    }
  }
  double del22 = C.delta * C.delta * (double)(1 << (2 * (k - 1)));
  double con1 = 1.5 * C.dt / del22 / C.norm;
  double con2 = -0.5 * C.dt / del22 / C.norm;
  ro[t] = rhs;
  return con1 * rhs + con2 * rold + rb;
}

// Grouped launches use a block map: block b covers elements
// [map[b].y, map[b].y + kBlockElems) of item map[b].x, so no block is spent on
// the parts of the grid a smaller case does not have.
__global__ void __launch_bounds__(256) k_rhs(const DevCase* __restrict__ cases, const LevelItem* __restrict__ items,
                                             const int2* __restrict__ bmap, int first_step) {
  const int2 bm = bmap[blockIdx.x];
  const LevelItem it = items[bm.x];
  const DevCase& C = cases[it.c];
  const int tend = min(C.ns, bm.y + kBlockElems);
  if (C.q0_const) {
    for (int t = bm.y + (int)threadIdx.x; t < tend; t += 256) C.rhsA[t] = rhs_value<true>(C, it, t, first_step);
  } else {
    for (int t = bm.y + (int)threadIdx.x; t < tend; t += 256) C.rhsA[t] = rhs_value<false>(C, it, t, first_step);
  }
}

// Split-precision form: the level update's right-hand side assembled to the
// solve's input in one pass over one 32 x 32 node tile per block,
//   b = norm * rhsA + (omega_k - nu_k C^T C omega_k)
// (the Crank-Nicolson form of operators.f90:126-130 with the explicit half of
// the diffusion applied by the 5-point stencil), written as FP64 (the
// refinement residual's right-hand side) and as three BF16 slices, row-major,
// through a shared-memory transpose. rhs_old = rhs as in k_rhs; rhsA itself
// is never stored.
//
// The kernel streams ~54 bytes per node and is bound by how many of them are
// in flight: each block first issues its whole input as asynchronous 8-byte
// copies into shared memory (omega with a one-node halo, the u and v faces
// the flux averages read, rhs_old), waits once, and then computes from shared
// memory (rhs_old, which each thread alone reads, straight into registers).
// Four resident blocks per SM (at most 64 registers a thread).
__device__ __forceinline__ double lap5_nodes(const double* __restrict__ x, int i, int j, int M, int N) {
  double c = x[i + (size_t)j * M];
  double s = 4.0 * c;
  if (i > 0) s -= x[i - 1 + (size_t)j * M];
  if (i + 1 < M) s -= x[i + 1 + (size_t)j * M];
  if (j > 0) s -= x[i + (size_t)(j - 1) * M];
  if (j + 1 < N) s -= x[i + (size_t)(j + 1) * M];
  return s;
}

__device__ __forceinline__ void split3_bf16(double x, uint16_t& s0, uint16_t& s1, uint16_t& s2) {
  __nv_bfloat16 a = __double2bfloat16(x);
  double r = x - (double)__bfloat162float(a);
  __nv_bfloat16 b = __double2bfloat16(r);
  r = r - (double)__bfloat162float(b);
  __nv_bfloat16 c = __double2bfloat16(r);
  s0 = __bfloat16_as_ushort(a);
  s1 = __bfloat16_as_ushort(b);
  s2 = __bfloat16_as_ushort(c);
}

__device__ __forceinline__ void cp_async8(void* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Stage a rows x cols window (origin r0, c0) of a column-major field with
// leading dimension ld and extents R x Cn into s[col][row] (row stride SP);
// entries outside the field are zero.
template <int SP>
__device__ __forceinline__ void stage_window(double* s, const double* __restrict__ f, int ld, int R, int Cn, int r0,
                                             int c0, int rows, int cols) {
  for (int e = threadIdx.x; e < rows * cols; e += blockDim.x) {
    const int a = e % rows, b = e / rows, r = r0 + a, c = c0 + b;
    double* d = s + b * SP + a;
    if (r >= 0 && r < R && c >= 0 && c < Cn) cp_async8(d, f + r + (size_t)c * ld);
    else *d = 0.0;
  }
}

struct RhsTile {
  double om[34][35];  // omega(i0 - 1 + a, j0 - 1 + b) at [b][a] (node coordinates, 0-based)
  double u[33][35];   // u face (i0 + a, j0 + b) at [b][a], a < 34 (face coordinates, 0-based)
  double v[34][34];   // v face (i0 + a, j0 + b) at [b][a], a < 33
  double t[32][33];   // the assembled b, [column][row]
};

__global__ void __launch_bounds__(256, 4) k_rhs_split(const DevCase* __restrict__ cases,
                                                   const LevelItem* __restrict__ items,
                                                   const RhsSplitDesc* __restrict__ sd,
                                                   const int2* __restrict__ bmap, int first_step) {
  const int2 bm = bmap[blockIdx.x];
  const LevelItem it = items[bm.x];
  const RhsSplitDesc& d = sd[bm.x];
  const DevCase& C = cases[it.c];
  const int m = C.m, n = C.n, M = m - 1, N = n - 1, k = it.k;
  const int ti = (M + 31) / 32;
  const int i0 = (bm.y % ti) * 32, j0 = (bm.y / ti) * 32;
  const double* om = C.omega + (size_t)(k - 1) * C.ns;
  __shared__ RhsTile S;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  if (!C.q0_const) {
    // general q0: direct loads
    for (int jj = ty; jj < 32; jj += 8) {
      const int i = i0 + tx, j = j0 + jj;
      double v = 0.0;
      if (i < M && j < N) {
        const int t = i + j * M;
        const double rA = rhs_value<false>(C, it, t, first_step);
        v = d.scale * rA;
        v = v + (om[t] - d.nu * lap5_nodes(om, i, j, M, N));
        d.b64[t] = v;
      }
      S.t[jj][tx] = v;
    }
  } else {
    const double* q = C.q + (size_t)(k - 1) * C.nq;
    const double* qv = q + (size_t)(m + 1) * n;
    double* ro = C.rhs_old + (size_t)(k - 1) * C.ns;
    const bool euler = first_step || *C.itime == 1;
    stage_window<35>(&S.om[0][0], om, M, M, N, i0 - 1, j0 - 1, 34, 34);
    stage_window<35>(&S.u[0][0], q, m + 1, m + 1, n, i0, j0, 34, 33);
    stage_window<34>(&S.v[0][0], qv, m, m, n + 1, i0, j0, 33, 34);
    // rhs_old of the thread's four nodes (read by no other thread): plain
    // loads into registers, in flight together with the tile copies
    const int la0 = tx, lr0 = 4 * ty;
    double ro4[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int ia = i0 + la0, jb = j0 + lr0 + r;
      ro4[r] = (!euler && ia < M && jb < N) ? ro[ia + (size_t)jb * M] : 0.0;
    }
    cp_async_all();
    __syncthreads();
    const double u0 = C.q0_u1 * (double)(1 << (k - 1));
    const double* bc = C.lastbc + (size_t)(k - 1) * C.nring;
    const int bottom = 2 * (n + 1), top = 2 * (n + 1) + m + 1, right = n + 1;
    const double del22 = C.delta * C.delta * (double)(1 << (2 * (k - 1)));
    const double vf = 0.5 * C.dt / C.re / del22 / C.norm;
    const double con1 = 1.5 * C.dt / del22 / C.norm;
    const double con2 = -0.5 * C.dt / del22 / C.norm;
    // Each thread walks four consecutive rows of one column of the tile and
    // keeps the values its next row shares with this one (the omega column,
    // the lower u faces, the v-face averages and fqu(j)) in registers. The
    // nonlinear term follows the reference's order (operators.f90:465-510,
    // :291-304) with q0 in closed form, as rhs_value<true>.
    const int la = tx, lb0 = 4 * ty;
    const int i = i0 + la + 2;  // reference (1-based) node index
    const bool iok = i - 2 < M;
    auto vrow = [&](int b) { return 0.5 * (S.v[b][la + 1] + S.v[b][la] + 0.0 + 0.0); };  // vavg(i, j0 + b + 1)
    double dn = S.om[lb0][la + 1], c = S.om[lb0 + 1][la + 1];
    double ul0 = S.u[lb0][la], ul1 = S.u[lb0][la + 1], ul2 = S.u[lb0][la + 2];
    double vb0 = vrow(lb0), vb1 = vrow(lb0 + 1);
    double fq_lo = 0.0;  // fqu(j - 1) = 0.5 (vavg(j) Wj(j) + vavg(j-1) Wj(j-1))
    {
      const int j = j0 + lb0 + 2;
      if (iok && j - 2 < N) fq_lo = 0.5 * (vb1 * c + vb0 * (j - 1 == 1 ? bc[bottom + i - 1] : dn));
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int lb = lb0 + r, j = j0 + lb + 2;
      const double up = S.om[lb + 2][la + 1], L = S.om[lb + 1][la], R = S.om[lb + 1][la + 2];
      const double uh0 = S.u[lb + 1][la], uh1 = S.u[lb + 1][la + 1], uh2 = S.u[lb + 1][la + 2];
      const double vb2 = vrow(lb + 2);
      if (!iok || j - 2 >= N) {
        S.t[lb][la] = 0.0;  // the K padding of the slices reads zero
      } else {
        const double WjU = j + 1 == n + 1 ? bc[top + i - 1] : up;
        const double fq_hi = 0.5 * (vb2 * WjU + vb1 * c);  // fqu(j)
        const double WiL = i - 1 == 1 ? bc[j - 1] : L;
        const double WiR = i + 1 == m + 1 ? bc[right + j - 1] : R;
        const double ua_m = 0.5 * (uh0 + ul0 + u0 + u0);  // uavg(i-1, j)
        const double ua_c = 0.5 * (uh1 + ul1 + u0 + u0);  // uavg(i, j)
        const double ua_p = 0.5 * (uh2 + ul2 + u0 + u0);  // uavg(i+1, j)
        const double fqv_i = -0.5 * (ua_p * WiR + ua_c * c);
        const double fqv_im = -0.5 * (ua_c * c + ua_m * WiL);
        const double rhs = fqv_i - fqv_im - fq_hi + fq_lo;
        fq_lo = fq_hi;
        const double rold = euler ? rhs : ro4[r];
        const int a = i - 1, b = j - 1;
        double rb = 0.0;
        if (a == 1 || a == m - 1 || b == 1 || b == n - 1) {
          rb = apply_bc_at(rb, a, b, m, n, vf, [&](int side, int I) { return ring_at(bc, m, n, side, I); });
          if (k < C.L) {
            const double* cr = C.omega + (size_t)k * C.ns;  // omega_{k+1}, already advanced
            rb = apply_bc_at(rb, a, b, m, n, vf,
                             [&](int side, int I) { return getbc_raw(cr, m, n, side, I) * 0.25; });
          } else {
            rb = apply_bc_at(rb, a, b, m, n, vf, [&](int, int) { return 0.0; });
          }
        }
        const int t = (i - 2) + (j - 2) * M;
        ro[t] = rhs;
        const double rA = con1 * rhs + con2 * rold + rb;
        // 5-point stencil of omega; the zero halo outside the grid drops the
        // boundary terms exactly as lap5_nodes does
        double s = 4.0 * c;
        s -= L;
        s -= R;
        s -= dn;
        s -= up;
        double v = d.scale * rA;
        v = v + (c - d.nu * s);
        d.b64[t] = v;
        S.t[lb][la] = v;
      }
      dn = c;
      c = up;
      ul0 = uh0; ul1 = uh1; ul2 = uh2;
      vb1 = vb2;
    }
  }
  __syncthreads();
  const int ii = threadIdx.x >> 3, g = threadIdx.x & 7;  // row ii, columns 4g .. 4g+3
  const int i = i0 + ii, j = j0 + 4 * g;
  if (i < M && j < N) {
    uint16_t a[4], b[4], c[4];
#pragma unroll
    for (int e = 0; e < 4; e++) split3_bf16(S.t[4 * g + e][ii], a[e], b[e], c[e]);
    // row stride and slice stride are multiples of 64 elements: 8-byte aligned
    // groups; columns >= N of the last group are zero (the K padding)
    uint16_t* o = d.Xs + (size_t)i * d.ld + j;
    auto st4 = [](uint16_t* p, const uint16_t* w) {
      uint2 u;
      u.x = (uint32_t)w[0] | ((uint32_t)w[1] << 16);
      u.y = (uint32_t)w[2] | ((uint32_t)w[3] << 16);
      *reinterpret_cast<uint2*>(p) = u;
    };
    st4(o, a);
    st4(o + d.sX, b);
    st4(o + 2 * d.sX, c);
  }
}

void launch_rhs_split(const DevCase* cases, const LevelItem* items, const RhsSplitDesc* sd, const int2* bmap,
                      int nblocks, int first, cudaStream_t st) {
  if (nblocks == 0) return;
  k_rhs_split<<<nblocks, 256, 0, st>>>(cases, items, sd, bmap, first);
}

// ---------------------------------------------------------------------------
// coarsify (operators.f90:307-333), in place on level k from level k-1.
__device__ __forceinline__ void coarsify_at(const DevCase& C, LevelItem it, int t) {
  int m = C.m, n = C.n;
  int ci = 3 * m / 4 - (m / 4 + 2) + 1;
  int i = t % ci + m / 4 + 2, j = t / ci + n / 4 + 2;
  int ii = 2 * i - m / 2 - 1, jj = 2 * j - n / 2 - 1;
  const double* f = C.omega + (size_t)(it.k - 2) * C.ns;
  double* c = C.omega + (size_t)(it.k - 1) * C.ns;
  auto R = [&](int x, int y) { return f[nidx(x, y, m)]; };
  c[nidx(i, j, m)] = R(ii, jj) + 0.50 * (R(ii - 1, jj) + R(ii + 1, jj) + R(ii, jj - 1) + R(ii, jj + 1)) +
                     0.25 * (R(ii - 1, jj - 1) + R(ii - 1, jj + 1) + R(ii + 1, jj - 1) + R(ii + 1, jj + 1));
}

__global__ void __launch_bounds__(256) k_coarsify(const DevCase* __restrict__ cases,
                                                  const LevelItem* __restrict__ items, const int2* __restrict__ bmap) {
  const int2 bm = bmap[blockIdx.x];
  const LevelItem it = items[bm.x];
  const DevCase& C = cases[it.c];
  const int tend = min(coarsify_count(C.m, C.n), bm.y + kBlockElems);
  for (int t = bm.y + (int)threadIdx.x; t < tend; t += 256) coarsify_at(C, it, t);
}

// ---------------------------------------------------------------------------
// curl (operators.f90:243-288) of s_k with sbc_k = get_bc(s_{k+1}, 1.0)
// (operators.f90:231; zero on the coarsest level, :218) into q_k.
// u face (i, j) (u = true) or v face (i, j) of level k, the reference's
// expressions in its order; x = s_k, cs = s_{k+1} (null on the coarsest level).
__device__ __forceinline__ double curl_face(bool u, int i, int j, int m, int n, const double* __restrict__ x,
                                            const double* __restrict__ cs) {
  auto xbc = [&](int side, int I) -> double { return cs ? getbc_raw(cs, m, n, side, I) * 1.0 : 0.0; };
  double v;
  if (u) {
    if (i == 1) v = xbc(SIDE_LEFT, j + 1) - xbc(SIDE_LEFT, j);
    else if (i == m + 1) v = xbc(SIDE_RIGHT, j + 1) - xbc(SIDE_RIGHT, j);
    else if (j == 1) v = x[nidx(i, 2, m)] - xbc(SIDE_BOTTOM, i);
    else if (j == n) v = xbc(SIDE_TOP, i) - x[nidx(i, n, m)];
    else v = x[nidx(i, j + 1, m)] - x[nidx(i, j, m)];
  } else {
    if (j == 1) v = xbc(SIDE_BOTTOM, i) - xbc(SIDE_BOTTOM, i + 1);
    else if (j == n + 1) v = xbc(SIDE_TOP, i) - xbc(SIDE_TOP, i + 1);
    else if (i == 1) v = -x[nidx(2, j, m)] + xbc(SIDE_LEFT, j);
    else if (i == m) v = -xbc(SIDE_RIGHT, j) + x[nidx(m, j, m)];
    else v = x[nidx(i, j, m)] - x[nidx(i + 1, j, m)];
  }
  return v;
}

// A thread's four faces (t, t + 256, t + 512, t + 768 of the level's face
// list: u faces column by column, then v faces) are all read before any is
// stored, so its loads of the four are in flight at once; the face's (i, j)
// comes from one division per thread, then by stepping 256 faces at a time.
__global__ void __launch_bounds__(256) k_curl(const DevCase* __restrict__ cases, const LevelItem* __restrict__ items,
                                              const int2* __restrict__ bmap) {
  static_assert(kBlockElems == 4 * 256, "four faces per thread");
  const int2 bm = bmap[blockIdx.x];
  const LevelItem it = items[bm.x];
  const DevCase& C = cases[it.c];
  const int m = C.m, n = C.n, k = it.k;
  const int tend = min(C.nq, bm.y + kBlockElems);
  const int nu = (m + 1) * n;
  const double* x = C.s + (size_t)(k - 1) * C.ns;
  const double* cs = (k < C.L) ? C.s + (size_t)k * C.ns : nullptr;
  int t = bm.y + (int)threadIdx.x;
  bool u = t < nu;
  int per = u ? m + 1 : m;
  int jq = (u ? t : t - nu) / per;
  int iq = (u ? t : t - nu) - jq * per;
  double v[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    v[r] = t < tend ? curl_face(u, iq + 1, jq + 1, m, n, x, cs) : 0.0;
    t += 256;
    iq += 256;
    while (iq >= per) {
      iq -= per;
      jq++;
    }
    if (u && t >= nu) {  // into the v faces
      u = false;
      per = m;
      jq = (t - nu) / per;
      iq = (t - nu) - jq * per;
    }
  }
  double* q = C.q + (size_t)(k - 1) * C.nq;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int tr = bm.y + (int)threadIdx.x + 256 * r;
    if (tr < tend) q[tr] = v[r];
  }
}

// ---------------------------------------------------------------------------
// vort = rot(reg(fb)) on level 1 (operators.f90:174 / :457, reg :513-528,
// rot :291-304). reg is gathered per face from the CSR-by-face table whose
// entries keep the reference's smear order.
__device__ __forceinline__ void regrot_at(const DevCase& C, int t) {
  int m = C.m, n = C.n;
  int i = t % (m - 1) + 2, j = t / (m - 1) + 2;
  const double* f = C.fb;
  double r = reg_face(C, f, voff(i, j, m, n)) - reg_face(C, f, voff(i - 1, j, m, n)) - reg_face(C, f, uoff(i, j, m)) +
             reg_face(C, f, uoff(i, j - 1, m));
  C.vort[t] = r;
}

__global__ void __launch_bounds__(256) k_regrot(const DevCase* __restrict__ cases, const int* __restrict__ cids,
                                                const int2* __restrict__ bmap) {
  const int2 bm = bmap[blockIdx.x];
  const DevCase& C = cases[cids[bm.x]];
  const int tend = min(C.ns, bm.y + kBlockElems);
  for (int t = bm.y + (int)threadIdx.x; t < tend; t += 256) regrot_at(C, t);
}

// Vertex fields of level k for the Tecplot export (write_tecplot,
// operators.f90:723-737), with del = 2^(k-1) delta and etf = reg(fb) on the
// level-1 faces (the reference uses it for every level), each in the
// reference's evaluation order:
//   u = 0.5 (q(u(i,j)) + q(u(i,j-1)) + q0(u(i,j)) + q0(u(i,j-1))) / del
//   v = 0.5 (q(v(i,j)) + q(v(i-1,j)) + q0(v(i,j)) + q0(v(i-1,j))) / del
//   etfx = delta (etf(u(i,j)) + etf(u(i,j-1))) / dt, etfy likewise on v
//   vort = omega(i,j,k) / del / del
// out: [5][(m-1)(n-1)], node (i,j) with i = 2..m fastest.
__global__ void k_vertex(const DevCase* __restrict__ cases, int c, int k, double* __restrict__ out) {
  const DevCase& C = cases[c];
  const int m = C.m, n = C.n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C.ns) return;
  const int i = t % (m - 1) + 2, j = t / (m - 1) + 2;
  const double fac = (double)(1 << (k - 1));
  const double del = fac * C.delta;
  const double* q = C.q + (size_t)(k - 1) * C.nq;
  const double* q0 = C.q0 + (size_t)(k - 1) * C.nq;
  const int u1 = uoff(i, j, m), u0 = uoff(i, j - 1, m), v1 = voff(i, j, m, n), v0 = voff(i - 1, j, m, n);
  out[t] = 0.5 * (q[u1] + q[u0] + q0[u1] + q0[u0]) / del;
  out[C.ns + t] = 0.5 * (q[v1] + q[v0] + q0[v1] + q0[v0]) / del;
  out[2 * (size_t)C.ns + t] = C.delta * (reg_face(C, C.fb, u1) + reg_face(C, C.fb, u0)) / C.dt;
  out[3 * (size_t)C.ns + t] = C.delta * (reg_face(C, C.fb, v1) + reg_face(C, C.fb, v0)) / C.dt;
  out[4 * (size_t)C.ns + t] = C.omega[(size_t)(k - 1) * C.ns + t] / del / del;
}

void launch_vertex(const DevCase* cases, int c, int k, int ns, double* out, cudaStream_t st) {
  k_vertex<<<(ns + 255) / 256, 256, 0, st>>>(cases, c, k, out);
}

// regT (operators.f90:531-546) of one face field, gathered per force in the
// reference's scatter order (ascending face index).
// motion = body velocity * delta - regT(q0(:,1));  rhsf = regT(q(:,1)) - motion
// (operators.f90:142-164, grid.f90:573-574).
__global__ void k_rhsf(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.y]];
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= C.nf) return;
  double mot = (C.bvel ? C.bvel[f] * C.delta : 0.0) - regT_force(C, C.q0, f);
  C.motion[f] = mot;
  C.rhsf[f] = regT_force(C, C.q, f) - mot;
  if (C.tq)  // (q + q0) at the force's faces, kept for the moving-body adjoint
    for (int p = 0; p < C.tcnt[f]; p++) {
      int fc = C.tface[f * 9 + p];
      C.tq[f * 9 + p] = C.q[fc] + C.q0[fc];
    }
}

// a_times output column: out = regT(q(:,1)) (operators.f90:461).
__global__ void k_regT_out(const DevCase* __restrict__ cases, const int* __restrict__ cids,
                           double* const* __restrict__ outs) {
  const DevCase& C = cases[cids[blockIdx.y]];
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= C.nf) return;
  outs[blockIdx.y][f] = regT_force(C, C.q, f);
}

// Unit right-hand side e_j for the a_times columns (operators.f90:50-52).
__global__ void k_unit_fb(const DevCase* __restrict__ cases, const int* __restrict__ cids, const int* __restrict__ cols) {
  const DevCase& C = cases[cids[blockIdx.y]];
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= C.nf) return;
  C.fb[f] = (f == cols[blockIdx.y]) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------
// Per-step outputs (write_force :583-659 with xg = fb/dt, write_circ :662-699,
// write_slip :549-580). Circulation is reduced in two fixed-order passes.
constexpr int kCircBlocks = 32;

__global__ void k_out_partial(const DevCase* __restrict__ cases, const LevelItem* __restrict__ items,
                              double* __restrict__ partial) {
  LevelItem it = items[blockIdx.y];
  const DevCase& C = cases[it.c];
  const double* om = C.omega + (size_t)(it.k - 1) * C.ns;
  double s = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < C.ns; t += gridDim.x * blockDim.x) s += om[t];
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = red[0];
}

__global__ void k_out_final(const DevCase* __restrict__ cases, const int* __restrict__ cids,
                            const int* __restrict__ item_base, const double* __restrict__ partial) {
  const DevCase& C = cases[cids[blockIdx.x]];
  int tid = threadIdx.x;
  double* out = C.out;
  // circulation per level
  if (tid < C.L) {
    int base = item_base[blockIdx.x] + tid;
    double s = 0.0;
    for (int b = 0; b < kCircBlocks; b++) s += partial[base * kCircBlocks + b];
    out[2 * C.nbody + tid] = s;
  }
  // forces per body: 2*delta * sum_f wsum_f * fb_f / dt
  __shared__ double fxs[64], fys[64];
  if (tid < 64) { fxs[tid] = 0.0; fys[tid] = 0.0; }
  __syncthreads();
  if (tid < C.nbody && tid < 64) {
    int body = C.bmin + tid;
    double sx = 0.0, sy = 0.0;
    for (int p = 0; p < C.nb; p++)
      if (C.bdyno[p] == body) {
        const double* ws = C.moving ? C.twsum : C.wsum;
        sx += ws[p] * (C.fb[p] / C.dt);
        sy += ws[C.nb + p] * (C.fb[C.nb + p] / C.dt);
      }
    out[tid] = sx * 2.0 * C.delta;
    out[C.nbody + tid] = sy * 2.0 * C.delta;
  }
  // slip = max |regT(q_1) - motion|
  __shared__ double mx[256];
  double s = 0.0;
  for (int f = tid; f < C.nf; f += blockDim.x) {
    double d = fabs(regT_force(C, C.q, f) - C.motion[f]);
    s = d > s ? d : s;
  }
  mx[tid] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (tid < w) mx[tid] = mx[tid] > mx[tid + w] ? mx[tid] : mx[tid + w];
    __syncthreads();
  }
  if (tid == 0) out[2 * C.nbody + C.L] = mx[0];
}

__global__ void k_step_begin(const DevCase* __restrict__ cases, int ncases) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncases) *cases[c].itime += 1;
}

// ---------------------------------------------------------------------------
// launchers
void launch_lastbc(const DevCase* cases, const LevelItem* items, int nitems, int max_ring, cudaStream_t st) {
  if (nitems == 0) return;
  dim3 g((max_ring + 255) / 256, nitems);
  k_lastbc<<<g, 256, 0, st>>>(cases, items);
}
std::vector<int2> block_map(const std::vector<int>& counts) {
  std::vector<int2> m;
  for (int i = 0; i < (int)counts.size(); i++)
    for (int f = 0; f < counts[i]; f += kBlockElems) m.push_back(make_int2(i, f));
  return m;
}
void launch_rhs(const DevCase* cases, const LevelItem* items, const int2* bmap, int nblocks, int first,
                cudaStream_t st) {
  if (nblocks == 0) return;
  k_rhs<<<nblocks, 256, 0, st>>>(cases, items, bmap, first);
}
void launch_coarsify(const DevCase* cases, const LevelItem* items, const int2* bmap, int nblocks, cudaStream_t st) {
  if (nblocks == 0) return;
  k_coarsify<<<nblocks, 256, 0, st>>>(cases, items, bmap);
}
void launch_curl(const DevCase* cases, const LevelItem* items, const int2* bmap, int nblocks, cudaStream_t st) {
  if (nblocks == 0) return;
  k_curl<<<nblocks, 256, 0, st>>>(cases, items, bmap);
}
void launch_regrot(const DevCase* cases, const int* cids, const int2* bmap, int nblocks, cudaStream_t st) {
  if (nblocks == 0) return;
  k_regrot<<<nblocks, 256, 0, st>>>(cases, cids, bmap);
}
void launch_rhsf(const DevCase* cases, const int* cids, int ncases, int max_nf, cudaStream_t st) {
  if (ncases == 0) return;
  dim3 g((max_nf + 127) / 128, ncases);
  k_rhsf<<<g, 128, 0, st>>>(cases, cids);
}
void launch_regT_out(const DevCase* cases, const int* cids, int ncases, int max_nf, double* const* outs,
                     cudaStream_t st) {
  if (ncases == 0) return;
  dim3 g((max_nf + 127) / 128, ncases);
  k_regT_out<<<g, 128, 0, st>>>(cases, cids, outs);
}
void launch_unit_fb(const DevCase* cases, const int* cids, const int* cols, int ncases, int max_nf,
                    cudaStream_t st) {
  if (ncases == 0) return;
  dim3 g((max_nf + 127) / 128, ncases);
  k_unit_fb<<<g, 128, 0, st>>>(cases, cids, cols);
}
void launch_outputs(const DevCase* cases, const LevelItem* items, int nitems, const int* cids, const int* item_base,
                    int ncases, double* partial, cudaStream_t st) {
  if (ncases == 0) return;
  dim3 g(kCircBlocks, nitems);
  k_out_partial<<<g, 256, 0, st>>>(cases, items, partial);
  k_out_final<<<ncases, 256, 0, st>>>(cases, cids, item_base, partial);
}
void launch_step_begin(const DevCase* cases, int ncases, cudaStream_t st) {
  k_step_begin<<<(ncases + 127) / 128, 128, 0, st>>>(cases, ncases);
}

}  // namespace ibfs
