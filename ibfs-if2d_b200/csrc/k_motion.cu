// k_motion.cu -- moving-body kernels: prescribed rigid pitching (move_body,
// grid.f90:523-576), the per-step regularisation rebuild (setup_reg,
// grid.f90:142-230) and the conjugate-gradient force solve (cjgr,
// operators.f90:393-441). All FP64.
//
// setup_reg for a moving body is rebuilt on the device every step into two
// fixed-capacity tables: per force, its <= 3x3 faces in ascending face index
// (the order of regT's scatter loop); per face of a fixed patch around the
// body's reach, its body points in ascending order (the order of reg's sum).
// Both use the reference's box test |x-xb| < 1.5 dx and the Roma-Peskin-Berger
// 3-point kernel.
#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"

namespace ibfs {

// Rigid pitching about (pivot_x, pivot_y): the body is the zero-pitch shape
// turned by -alpha(t) (the sign convention of line(), grid.f90:442), with
// alpha(t) = amp sin(omega t), t = itime dt; body velocity = rotation rate x r.
__global__ void k_move_body(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.y]];
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= C.nb) return;
  double t = C.dt * (double)(*C.itime);
  double al = C.pitch_amp * sin(C.pitch_omega * t);
  double ald = C.pitch_amp * C.pitch_omega * cos(C.pitch_omega * t);
  double th = -al, thd = -ald;
  double c = cos(th), s = sin(th);
  double rx = C.xb0[k] - C.pivot_x, ry = C.yb0[k] - C.pivot_y;
  double x = C.pivot_x + c * rx - s * ry;
  double y = C.pivot_y + s * rx + c * ry;
  C.xb[k] = x;
  C.yb[k] = y;
  C.bvel[k] = -thd * (y - C.pivot_y);
  C.bvel[C.nb + k] = thd * (x - C.pivot_x);
}

// Actuator jets (actuation, grid.f90:579-605; u_jet, :608-633): point
// nb - nact + p gets the velocity u_jet = (u_j + u_j_osc sin(omg_j dt itime))
// times (cos, sin)(pi/180 theta_j) of its actuator, after move_body; rhsf
// multiplies it by delta as the reference's motion does. The parameters are
// read once instead of from input/actuator.NNN.inp every step.
__global__ void k_actuate(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.y]];
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= C.nact) return;
  const double* a = C.act + 5 * p;
  int k = C.nb - C.nact + p;
  double u = a[0] + a[1] * sin(a[2] * C.dt * (double)(*C.itime));
  C.bvel[k] = u * a[3];
  C.bvel[C.nb + k] = u * a[4];
}

// Per-force table: u faces at (dx(i-1)-ox, dx(j-1)-oy+dx/2), v faces at
// (dx(i-1)-ox+dx/2, dx(j-1)-oy); candidates scanned j-major for ascending
// face index.
__global__ void k_setup_reg_force(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.y]];
  const double ox = C.offx, oy = C.offy;
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= C.nf) return;
  int m = C.m, n = C.n, nb = C.nb;
  bool vcomp = f >= nb;
  int k = vcomp ? f - nb : f;
  double dx = C.delta, d2 = 0.5 * dx, sup = 3.0 * d2;
  double xk = C.xb[k], yk = C.yb[k];
  double sx = vcomp ? d2 : 0.0, sy = vcomp ? 0.0 : d2;
  int ic = (int)floor((xk + ox - sx) / dx) + 1, jc = (int)floor((yk + oy - sy) / dx) + 1;
  int imax = vcomp ? m : m + 1, jmax = vcomp ? n + 1 : n;
  int cnt = 0;
  double ws = 0.0;
  for (int j = jc - 2; j <= jc + 2; j++) {
    if (j < 1 || j > jmax) continue;
    for (int i = ic - 2; i <= ic + 2; i++) {
      if (i < 1 || i > imax) continue;
      double x = dx * (double)(i - 1) - ox + sx;
      double y = dx * (double)(j - 1) - oy + sy;
      if (fabs(x - xk) < sup && fabs(y - yk) < sup && cnt < 9) {
        double w = (dx * dx) * deltafnc_d(x, xk, dx) * deltafnc_d(y, yk, dx);
        C.tface[f * 9 + cnt] = vcomp ? (m + 1) * n + (i - 1) + (j - 1) * m : (i - 1) + (j - 1) * (m + 1);
        C.tw[f * 9 + cnt] = w;
        ws += w;
        cnt++;
      }
    }
  }
  C.tcnt[f] = cnt;
  C.twsum[f] = ws;
}

// Per-face table over the patch: body points in ascending order.
__global__ void k_setup_reg_patch(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.y]];
  const double ox = C.offx, oy = C.offy;
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  int nu_p = C.pu_w * C.pu_h, np = nu_p + C.pv_w * C.pv_h;
  if (p >= np) return;
  double dx = C.delta, d2 = 0.5 * dx, sup = 3.0 * d2;
  bool vcomp = p >= nu_p;
  int i, j;
  if (!vcomp) { i = p % C.pu_w + C.pu_i0; j = p / C.pu_w + C.pu_j0; }
  else { int q = p - nu_p; i = q % C.pv_w + C.pv_i0; j = q / C.pv_w + C.pv_j0; }
  double x = dx * (double)(i - 1) - ox + (vcomp ? d2 : 0.0);
  double y = dx * (double)(j - 1) - oy + (vcomp ? 0.0 : d2);
  int cnt = 0;
  for (int k = 0; k < C.nb; k++) {
    double xk = C.xb[k], yk = C.yb[k];
    if (fabs(x - xk) < sup && fabs(y - yk) < sup) {
      if (cnt < kPatchCap) {
        C.pf[p * kPatchCap + cnt] = vcomp ? C.nb + k : k;
        C.pw[p * kPatchCap + cnt] = (dx * dx) * deltafnc_d(x, xk, dx) * deltafnc_d(y, yk, dx);
      } else {
        atomicOr(C.status, 4);  // patch capacity exceeded
      }
      cnt++;
    }
  }
  C.pcnt[p] = cnt < kPatchCap ? cnt : kPatchCap;
}

// --------------------------------------------------------------------------
// CG (operators.f90:393-441), one CTA per case, FP64 reductions in a fixed
// order (block tree). Scalars: sc[0] delta_new, sc[1] delta_old, sc[2] eps,
// sc[3] alpha, sc[4] r.r of the preconditioned form; it[0] iterations,
// it[1] active.
__device__ double block_dot(const double* a, const double* b, int n, double* red) {
  double s = 0.0;
  for (int t = threadIdx.x; t < n; t += blockDim.x) s = fma(a[t], b[t], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

// z = P r = Q Lk^-T Lk^-1 Q^T r (one CTA): the force operator factored at the
// body turned by the grid angle theta_k nearest to this step's pitch
// (A_k = Lk Lk^T; slot k of pre_fac holds Lk^-1 and its transpose, row-major),
// applied in that slot's frame. A rigid rotation moves every point's force
// pair with it, so A(theta) ~ Q A_k Q^T up to the grid's anisotropy, Q the
// rotation by theta - theta_k of each (fx_k, fy_k); theta = 0 for a body that
// does not move (one slot). The triangular products run one warp per row, in
// a fixed order.
__device__ void cg_precond(const DevCase& C, const double* __restrict__ r, double* __restrict__ z) {
  const int nb = C.nb, nf = C.nf;
  const int slot = *C.pre_idx;
  const double* __restrict__ Linv = C.pre_fac + (size_t)slot * 2 * nf * nf;
  const double* __restrict__ LinvT = Linv + (size_t)nf * nf;
  double c = 1.0, s = 0.0;
  if (C.moving) {
    double th = -(C.pitch_amp * sin(C.pitch_omega * (C.dt * (double)(*C.itime))));
    th = th - (double)(slot - C.pre_k0) * C.pre_dth;
    c = cos(th);
    s = sin(th);
  }
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {  // Q^T r
    double rx = r[k], ry = r[nb + k];
    z[k] = c * rx + s * ry;
    z[nb + k] = -s * rx + c * ry;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double* y = C.cg_y;
  for (int row = warp; row < nf; row += nw) {  // y = L0^-1 (Q^T r)
    const double* Mr = Linv + (size_t)row * nf;
    double a = 0.0;
    for (int k = lane; k <= row; k += 32) a = fma(Mr[k], z[k], a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) y[row] = a;
  }
  __syncthreads();
  for (int row = warp; row < nf; row += nw) {  // L0^-T y
    const double* Mr = LinvT + (size_t)row * nf;
    double a = 0.0;
    for (int k = row + lane; k < nf; k += 32) a = fma(Mr[k], y[k], a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) z[row] = a;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {  // Q (...)
    double wx = z[k], wy = z[nb + k];
    z[k] = c * wx - s * wy;
    z[nb + k] = s * wx + c * wy;
  }
  __syncthreads();
}

// r = b - A x (A x in cg_q), d = r, delta_new = r.r, eps, active
// (preconditioned: z = P r, d = z, delta_new = r.z; the stop test stays r.r).
__global__ void k_cg_start(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.x]];
  __shared__ double red[256];
  int nf = C.nf;
  if (C.cg_pre) {
    for (int t = threadIdx.x; t < nf; t += blockDim.x) C.cg_r[t] = C.rhsf[t] - C.cg_q[t];
    __syncthreads();
    double rr = block_dot(C.cg_r, C.cg_r, nf, red);
    cg_precond(C, C.cg_r, C.cg_z);
    for (int t = threadIdx.x; t < nf; t += blockDim.x) C.cg_d[t] = C.cg_z[t];
    double rz = block_dot(C.cg_r, C.cg_z, nf, red);
    double eps = C.cgtol * C.cgtol;
    if (C.cg_rel) eps = eps * block_dot(C.rhsf, C.rhsf, nf, red);
    if (threadIdx.x == 0) {
      C.cg_sc[0] = rz;
      C.cg_sc[2] = eps;
      C.cg_sc[4] = rr;
      C.cg_it[0] = 0;
      C.cg_it[1] = (C.cg_max_iter > 0 && rr > eps) ? 1 : 0;
    }
    return;
  }
  for (int t = threadIdx.x; t < nf; t += blockDim.x) {
    double r = C.rhsf[t] - C.cg_q[t];
    C.cg_r[t] = r;
    C.cg_d[t] = r;
  }
  __syncthreads();
  double dn = block_dot(C.cg_r, C.cg_r, nf, red);
  double eps = C.cgtol * C.cgtol;
  if (C.cg_rel) eps = eps * block_dot(C.rhsf, C.rhsf, nf, red);
  if (threadIdx.x == 0) {
    C.cg_sc[0] = dn;
    C.cg_sc[2] = eps;
    C.cg_it[0] = 0;
    C.cg_it[1] = (C.cg_max_iter > 0 && dn > eps) ? 1 : 0;
  }
}

// alpha = delta_new / d.q ; x += alpha d ; r -= alpha q unless it is recomputed.
__global__ void k_cg_alpha(const DevCase* __restrict__ cases, const int* __restrict__ cids, int recompute) {
  const DevCase& C = cases[cids[blockIdx.x]];
  if (!C.cg_it[1]) return;
  __shared__ double red[256];
  int nf = C.nf;
  double dq = block_dot(C.cg_d, C.cg_q, nf, red);
  double alpha = C.cg_sc[0] / dq;
  for (int t = threadIdx.x; t < nf; t += blockDim.x) {
    C.fb[t] = C.fb[t] + alpha * C.cg_d[t];
    if (!recompute) C.cg_r[t] = C.cg_r[t] - alpha * C.cg_q[t];
  }
  if (threadIdx.x == 0) C.cg_sc[3] = alpha;
}

// r = b - A x with A x in cg_q2 (every 50th iteration, operators.f90:421-422).
__global__ void k_cg_resid(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.x]];
  if (!C.cg_it[1]) return;
  for (int t = threadIdx.x; t < C.nf; t += blockDim.x) C.cg_r[t] = C.rhsf[t] - C.cg_q2[t];
}

// delta_old = delta_new; delta_new = r.r; d = r + beta d; iter++; active
// (preconditioned: z = P r, delta_new = r.z, d = z + beta d, stop on r.r).
__global__ void k_cg_beta(const DevCase* __restrict__ cases, const int* __restrict__ cids) {
  const DevCase& C = cases[cids[blockIdx.x]];
  if (!C.cg_it[1]) return;
  __shared__ double red[256];
  int nf = C.nf;
  if (C.cg_pre) {
    double rr = block_dot(C.cg_r, C.cg_r, nf, red);
    cg_precond(C, C.cg_r, C.cg_z);
    double rz = block_dot(C.cg_r, C.cg_z, nf, red);
    double beta = rz / C.cg_sc[0];
    for (int t = threadIdx.x; t < nf; t += blockDim.x) C.cg_d[t] = C.cg_z[t] + beta * C.cg_d[t];
    __syncthreads();
    if (threadIdx.x == 0) {
      C.cg_sc[1] = C.cg_sc[0];
      C.cg_sc[0] = rz;
      C.cg_sc[4] = rr;
      int it = C.cg_it[0] + 1;
      C.cg_it[0] = it;
      C.cg_it[1] = (it < C.cg_max_iter && rr > C.cg_sc[2]) ? 1 : 0;
    }
    return;
  }
  double dn = block_dot(C.cg_r, C.cg_r, nf, red);
  double beta = dn / C.cg_sc[0];
  for (int t = threadIdx.x; t < nf; t += blockDim.x) C.cg_d[t] = C.cg_r[t] + beta * C.cg_d[t];
  __syncthreads();
  if (threadIdx.x == 0) {
    C.cg_sc[1] = C.cg_sc[0];
    C.cg_sc[0] = dn;
    int it = C.cg_it[0] + 1;
    C.cg_it[0] = it;
    C.cg_it[1] = (it < C.cg_max_iter && dn > C.cg_sc[2]) ? 1 : 0;
  }
}

// Copy a face field (the a_times input vector) into a shadow's fb.
__global__ void k_copy_vec(double* const* __restrict__ dst, const double* const* __restrict__ src,
                           const int* __restrict__ n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n[blockIdx.y]) dst[blockIdx.y][i] = src[blockIdx.y][i];
}

void launch_move_body(const DevCase* cases, const int* cids, int ncases, int max_nb, cudaStream_t st) {
  if (ncases) k_move_body<<<dim3((max_nb + 127) / 128, ncases), 128, 0, st>>>(cases, cids);
}
void launch_actuate(const DevCase* cases, const int* cids, int ncases, int max_nact, cudaStream_t st) {
  if (ncases) k_actuate<<<dim3((max_nact + 127) / 128, ncases), 128, 0, st>>>(cases, cids);
}
void launch_setup_reg_moving(const DevCase* cases, const int* cids, int ncases, int max_nf, int max_patch,
                             cudaStream_t st) {
  if (!ncases) return;
  k_setup_reg_force<<<dim3((max_nf + 127) / 128, ncases), 128, 0, st>>>(cases, cids);
  k_setup_reg_patch<<<dim3((max_patch + 127) / 128, ncases), 128, 0, st>>>(cases, cids);
}
void launch_cg_start(const DevCase* cases, const int* cids, int ncases, cudaStream_t st) {
  if (ncases) k_cg_start<<<ncases, 256, 0, st>>>(cases, cids);
}
void launch_cg_alpha(const DevCase* cases, const int* cids, int ncases, int recompute, cudaStream_t st) {
  if (ncases) k_cg_alpha<<<ncases, 256, 0, st>>>(cases, cids, recompute);
}
void launch_cg_resid(const DevCase* cases, const int* cids, int ncases, cudaStream_t st) {
  if (ncases) k_cg_resid<<<ncases, 256, 0, st>>>(cases, cids);
}
void launch_cg_beta(const DevCase* cases, const int* cids, int ncases, cudaStream_t st) {
  if (ncases) k_cg_beta<<<ncases, 256, 0, st>>>(cases, cids);
}
void launch_copy_vec(double* const* dst, const double* const* src, const int* n, int nvec, int max_n,
                     cudaStream_t st) {
  if (nvec) k_copy_vec<<<dim3((max_n + 127) / 128, nvec), 128, 0, st>>>(dst, src, n);
}

}  // namespace ibfs
