// k_adjoint.cu -- kernels of the discrete adjoint of one IBFS advance.
//
// The forward step (operators.f90:62-188, stationary body, Cholesky solve) is
// linear in every operator except the bilinear convective term; its adjoint
// runs the transposed operators in reverse order:
//   curl^T   = (rot on the nodes, ring terms)     (curl, operators.f90:243-288)
//   rot^T    = curl with a zero ring              (rot,  operators.f90:291-304)
//   get_bc^T : ring -> box-perimeter nodes        (get_bc, operators.f90:336-367)
//   apply_bc^T: edge nodes -> ring                (apply_bc, operators.f90:370-390)
//   coarsify^T: coarse centre -> fine nodes       (coarsify, operators.f90:307-333)
//   reg^T = regT, regT^T = reg                    (operators.f90:513-546)
//   nonlinear: transposed linearisation about the stored forward state
// The DST-based inverses (ctci, ainv, the CN update) are symmetric and reuse
// the forward sine-transform GEMMs; the Cholesky solve is symmetric too.
// All kernels are gathers (no atomics), so the adjoint is deterministic.
//
// Every kernel serves a group of slots (cases differentiated together): slot
// blockIdx.z is case cids[slot] with working set adj[slot]; grids are sized by
// the group's largest case and a slot skips levels beyond its own L.
#include "ibfs_adjoint.cuh"

namespace ibfs {

__device__ __forceinline__ int ring_off(int m, int n, int side) {
  return side == SIDE_LEFT ? 0 : side == SIDE_RIGHT ? n + 1 : side == SIDE_BOTTOM ? 2 * (n + 1) : 2 * (n + 1) + m + 1;
}

// (s_hat, sbc_hat) = curl^T(q_hat) on level k; zero when k > nlev.
__global__ void k_adj_curlT(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids, int nlev,
                            int use_q1) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  int k = blockIdx.y + 1;
  if (k > C.L) return;
  int m = C.m, n = C.n;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double* Q = use_q1 ? A.aQ1 : A.aQ + (size_t)(k - 1) * C.nq;
  double* S = A.aS + (size_t)(k - 1) * C.ns;
  double* R = A.aSbc + (size_t)(k - 1) * C.nring;
  auto qu = [&](int i, int j) { return Q[uoff(i, j, m)]; };
  auto qv = [&](int i, int j) { return Q[voff(i, j, m, n)]; };
  if (t < C.ns) {
    if (k > nlev) { S[t] = 0.0; return; }
    int i = t % (m - 1) + 2, j = t / (m - 1) + 2;
    S[t] = qv(i, j) - qv(i - 1, j) - qu(i, j) + qu(i, j - 1);
  } else if (t < C.ns + C.nring) {
    int r = t - C.ns;
    if (k > nlev) { R[r] = 0.0; return; }
    double v = 0.0;
    if (r < n + 1) {  // left, J = r+1
      int J = r + 1;
      if (J >= 2) v += qu(1, J - 1);
      if (J <= n) v -= qu(1, J);
      if (J >= 2 && J <= n) v += qv(1, J);
    } else if (r < 2 * (n + 1)) {  // right
      int J = r - (n + 1) + 1;
      if (J >= 2) v += qu(m + 1, J - 1);
      if (J <= n) v -= qu(m + 1, J);
      if (J >= 2 && J <= n) v -= qv(m, J);
    } else if (r < 2 * (n + 1) + m + 1) {  // bottom, I
      int I = r - 2 * (n + 1) + 1;
      if (I >= 2 && I <= m) v -= qu(I, 1);
      if (I <= m) v += qv(I, 1);
      if (I >= 2) v -= qv(I - 1, 1);
    } else {  // top
      int I = r - 2 * (n + 1) - (m + 1) + 1;
      if (I >= 2 && I <= m) v += qu(I, n);
      if (I <= m) v += qv(I, n + 1);
      if (I >= 2) v -= qv(I - 1, n + 1);
    }
    R[r] = v;
  }
}

// apply_bc^T (fac) of a node field into a ring: entry side+I collects the edge
// node apply_bc adds it to (operators.f90:382-389).
__device__ __forceinline__ double applybcT_at(const double* __restrict__ x, int m, int n, int r) {
  auto X = [&](int a, int b) { return x[ridx(a, b, m)]; };
  if (r < n + 1) { int J = r + 1; return (J >= 2 && J <= n) ? X(1, J - 1) : 0.0; }
  if (r < 2 * (n + 1)) { int J = r - (n + 1) + 1; return (J >= 2 && J <= n) ? X(m - 1, J - 1) : 0.0; }
  if (r < 2 * (n + 1) + m + 1) { int I = r - 2 * (n + 1) + 1; return (I >= 2 && I <= m) ? X(I - 1, 1) : 0.0; }
  int I = r - 2 * (n + 1) - (m + 1) + 1;
  return (I >= 2 && I <= m) ? X(I - 1, n - 1) : 0.0;
}

// get_bc^T: the value gathered by coarse node r(a,b) (1-based) from a ring,
// each ring entry having taken 1 x or 0.5 x of that node (operators.f90:348-366).
__device__ __forceinline__ double getbcT_at(const double* __restrict__ ring, int m, int n, int a, int b) {
  double v = 0.0;
  int bot = 2 * (n + 1), top = bot + m + 1, right = n + 1;
  if (b == n / 4 || b == 3 * n / 4) {
    int off = b == n / 4 ? bot : top;
    int u = a - m / 4;
    if (u >= 0 && u <= m / 2) {
      int te = 2 * u;  // even entry t = te
      v += ring[off + te];
      if (te - 1 >= 1) v += 0.5 * ring[off + te - 1];
      if (te + 1 <= m - 1) v += 0.5 * ring[off + te + 1];
    }
  }
  if (a == m / 4 || a == 3 * m / 4) {
    int off = a == m / 4 ? 0 : right;
    int u = b - n / 4;
    if (u >= 0 && u <= n / 2) {
      int te = 2 * u;
      v += ring[off + te];
      if (te - 1 >= 1) v += 0.5 * ring[off + te - 1];
      if (te + 1 <= n - 1) v += 0.5 * ring[off + te + 1];
    }
  }
  return v;
}

// aW_k += v ; sbc_hat_k += apply_bc^T(v) (vort2flux adjoint, one level).
__global__ void k_adj_v2f_level(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids, int k) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  if (k > C.L) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double* v = A.aZ1;
  if (t < C.ns) {
    A.aW[(size_t)(k - 1) * C.ns + t] += v[t];
  } else if (t < C.ns + C.nring) {
    int r = t - C.ns;
    A.aSbc[(size_t)(k - 1) * C.nring + r] += applybcT_at(v, C.m, C.n, r);
  }
}

// dst(a, b) += fac * get_bc^T(ring) on the box perimeter of a node field, for
// the three uses of the adjoint (level k < L of the slot):
//   GETBC_SBC  ring aSbc_k -> aS_{k+1}  (vort2flux, fac 1)
//   GETBC_OBC  ring aObc   -> aW_{k+1}  (omega_bc of the CN update, fac 0.25)
//   GETBC_LB   ring aLb_k  -> aW2_{k+1} (lastbc, fac 0.25)
__global__ void k_adj_getbcT(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj,
                             const int* __restrict__ cids, int which, int k, double fac) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  if (k >= C.L) return;
  const double* ring = which == GETBC_SBC ? A.aSbc + (size_t)(k - 1) * C.nring
                     : which == GETBC_OBC ? A.aObc : A.aLb + (size_t)(k - 1) * C.nring;
  double* dst = (which == GETBC_SBC ? A.aS : which == GETBC_OBC ? A.aW : A.aW2) + (size_t)k * C.ns;
  int m = C.m, n = C.n;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  // perimeter nodes of the box [m/4,3m/4] x [n/4,3n/4]: bottom/top rows, then left/right columns
  int wa = m / 2 + 1, hb = n / 2 + 1;
  int a, b;
  if (t < 2 * wa) { a = m / 4 + t % wa; b = t < wa ? n / 4 : 3 * n / 4; }
  else if (t < 2 * wa + 2 * (hb - 2)) {
    int u = t - 2 * wa;
    a = u < hb - 2 ? m / 4 : 3 * m / 4;
    b = n / 4 + 1 + u % (hb - 2);
  } else return;
  dst[ridx(a, b, m)] += fac * getbcT_at(ring, m, n, a, b);
}

// coarsify^T (operators.f90:320-332): fine level k-1 gathers the coarse
// centre of level k with the full-weighting weights; then the centre of
// level k is cleared (it was overwritten in the forward pass).
__global__ void k_adj_coarsifyT(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids, int k) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  if (k > C.L) return;
  int m = C.m, n = C.n;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C.ns) return;
  int ii = t % (m - 1) + 2, jj = t / (m - 1) + 2;
  const double* Wc = A.aW + (size_t)(k - 1) * C.ns;
  double s = 0.0;
  // coarse i with |ii - (2i - m/2 - 1)| <= 1, i in [m/4+2, 3m/4]
  for (int di = -1; di <= 1; di++) {
    int x2 = ii + m / 2 + 1 + di;  // = 2i
    if (x2 & 1) continue;
    int i = x2 / 2;
    if (i < m / 4 + 2 || i > 3 * m / 4) continue;
    double wi = di == 0 ? 1.0 : 0.5;
    for (int dj = -1; dj <= 1; dj++) {
      int y2 = jj + n / 2 + 1 + dj;
      if (y2 & 1) continue;
      int j = y2 / 2;
      if (j < n / 4 + 2 || j > 3 * n / 4) continue;
      double wj = dj == 0 ? 1.0 : 0.5;
      s += wi * wj * Wc[nidx(i, j, m)];
    }
  }
  A.aW[(size_t)(k - 2) * C.ns + t] += s;
}

__global__ void k_adj_zero_centre(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids, int k) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  if (k > C.L) return;
  int m = C.m, n = C.n;
  int ci = 3 * m / 4 - (m / 4 + 2) + 1, cj = 3 * n / 4 - (n / 4 + 2) + 1;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ci * cj) return;
  int i = t % ci + m / 4 + 2, j = t / ci + n / 4 + 2;
  A.aW[(size_t)(k - 1) * C.ns + nidx(i, j, m)] = 0.0;
}

// curl(x, 0) at one face (rot^T of a node field, operators.f90:243-288 with a
// zero ring).
__device__ __forceinline__ double curl0_face(const double* __restrict__ x, int m, int n, int face) {
  auto X = [&](int i, int j) { return (i >= 2 && i <= m && j >= 2 && j <= n) ? x[nidx(i, j, m)] : 0.0; };
  int nu = (m + 1) * n;
  if (face < nu) {
    int i = face % (m + 1) + 1, j = face / (m + 1) + 1;
    return (i == 1 || i == m + 1) ? 0.0 : X(i, j + 1) - X(i, j);
  }
  int fv = face - nu, i = fv % m + 1, j = fv / m + 1;
  return (j == 1 || j == n + 1) ? 0.0 : X(i, j) - X(i + 1, j);
}

// regT(curl(x, 0)) for one force, gathered over the force's faces.
__device__ __forceinline__ double regT_curl0(const DevCase& C, const double* __restrict__ x, int f) {
  double s = 0.0;
  if (C.moving) {
    for (int p = 0; p < C.tcnt[f]; p++) s += C.tw[f * 9 + p] * curl0_face(x, C.m, C.n, C.tface[f * 9 + p]);
    return s;
  }
  for (int q = C.force_ptr[f]; q < C.force_ptr[f + 1]; q++) s += C.force_w[q] * curl0_face(x, C.m, C.n, C.force_face[q]);
  return s;
}

// F_hat' = objective term + (-regT(curl0(aZ1))) (projection adjoint,
// operators.f90:174) ; objective: J += wx_b fx_b + wy_b fy_b with
// f = 2 delta / dt * sum wsum_f fb_f (write_force; a moving body's wsum is
// the sum of its current weights).
__global__ void k_adj_force(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= C.nf) return;
  int p = f < C.nb ? f : f - C.nb;
  int b = C.bdyno[p] - C.bmin;
  double w = f < C.nb ? A.wx[b] : A.wy[b];
  double v = w * 2.0 * C.delta / C.dt * (C.moving ? C.twsum[f] : C.wsum[f]);
  A.aF[f] = v - regT_curl0(C, A.aZ1, f);
}

// aTmp = Linv aF (lower) / aRf = LinvT aTmp (upper) on adjoint vectors; warp per row.
__global__ void k_adj_tri(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj,
                          const int* __restrict__ cids, int upper) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  const double* in = upper ? A.aTmp : A.aF;
  double* out = upper ? A.aRf : A.aTmp;
  int nf = C.nf;
  int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (row >= nf) return;
  const double* Mr = (upper ? C.LinvT : C.Linv) + (size_t)row * nf;
  int k0 = upper ? row : 0, k1 = upper ? nf : row + 1;
  double s = 0.0;
  for (int k = k0 + lane; k < k1; k += 32) s = fma(Mr[k], in[k], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[row] = s;
}

// q1_hat = reg(rhsf_hat) on all faces; grad_vel -= delta * rhsf_hat
// (rhsf = regT(q1) - (delta*vel - regT(q0)), operators.f90:155-164).
__global__ void k_adj_rhsf(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < C.nq) A.aQ1[t] = reg_face(C, A.aRf, t);
  if (t < C.nf) A.aGrad[t] -= C.delta * A.aRf[t];
}

// ---------------------------------------------------------------------------
// Moving body (rigid pitching, CG force solve). The force operator
// A = regT M reg (M = curl vort2flux_1 ainv rot, a_times, operators.f90:444-462)
// is solved by CG in the forward step; its adjoint needs A^T = regT M^T reg,
// applied with the transposed operators above, and the derivative of the
// smearing weights with respect to the body positions.

// aQ1 = reg(x) on all faces (the first operator of A^T).
__global__ void k_adjm_reg_in(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids,
                              const double* const* __restrict__ xs) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < C.nq) A.aQ1[t] = reg_face(C, xs[slot], t);
}

// out = regT(curl(aZ1, 0)) (the last two operators of A^T).
__global__ void k_adjm_regT_curl0(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids,
                                  double* const* __restrict__ outs) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < C.nf) outs[slot][f] = regT_curl0(C, A.aZ1, f);
}

// One step's contribution to dJ/d(pitch amplitude, radians), added to *acc.
// The weight w(face, f) = dx^2 delta(x_face - X_k) delta(y_face - Y_k) of force
// f (component of body point k) enters the step through
//   rhsf  = regT(q1 + q0) - dx V          (b-hat = rhsf_hat = aRf)
//   fb    = A^-1 rhsf, A = regT M reg     (u = M reg fb, v = M^T reg b-hat)
//   omega_1 -= ainv rot reg fb            (g = curl0(ainv omega_1-hat) = curl0(aZ1))
//   fx_b  = 2 dx / dt sum_f fb_f sum_face w(face, f)
// so dJ/dw(face, f) = b-hat_f (q1 + q0 - u)_face - fb_f (g + v)_face
//                     + 2 dx / dt wobj_f fb_f,
// and dJ/dX_k = sum over both components and their faces of dw/dX_k times it.
// With alpha = A sin(Om t), theta = -alpha about the pivot:
//   dX/dA = (Y - py) sin(Om t), dY/dA = -(X - px) sin(Om t),
//   V = thetadot (-(Y - py), X - px), thetadot = -A Om cos(Om t),
//   dV/dA from both d thetadot/dA = -Om cos(Om t) and dX/dA, dY/dA;
// the velocity enters rhsf as -dx V, so dJ/dV_f = -dx b-hat_f.
// One block; the points are reduced in a fixed order.
__global__ void k_adjm_position(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids,
                                const AdjCase* __restrict__ acg, const double* const* __restrict__ us,
                                double* __restrict__ accs) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  const double* __restrict__ zcg = acg[slot].aZ1;
  const double* __restrict__ u = us[slot];
  double* acc = accs + slot;
  const int m = C.m, n = C.n, nb = C.nb;
  const double dx = C.delta, d2 = 0.5 * dx;
  const double t = C.dt * (double)(*C.itime);
  const double sn = sin(C.pitch_omega * t), cs = cos(C.pitch_omega * t);
  const double thd = -C.pitch_amp * C.pitch_omega * cs;
  double part = 0.0;
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    const double X = C.xb[k], Y = C.yb[k];
    const int b = C.bdyno[k] - C.bmin;
    double gx = 0.0, gy = 0.0;
    for (int comp = 0; comp < 2; comp++) {
      const int f = comp ? nb + k : k;
      const double sx = comp ? d2 : 0.0, sy = comp ? 0.0 : d2;
      const double fbf = C.fb[f], bh = A.aRf[f];
      const double wobj = (comp ? A.wy[b] : A.wx[b]) * 2.0 * dx / C.dt * fbf;
      for (int p = 0; p < C.tcnt[f]; p++) {
        const int face = C.tface[f * 9 + p];
        int i, j;
        if (!comp) {
          i = face % (m + 1) + 1;
          j = face / (m + 1) + 1;
        } else {
          int fv = face - (m + 1) * n;
          i = fv % m + 1;
          j = fv / m + 1;
        }
        const double x = dx * (double)(i - 1) - C.offx + sx;
        const double y = dx * (double)(j - 1) - C.offy + sy;
        const double G = bh * (A.tq[f * 9 + p] - u[face]) -
                         fbf * (curl0_face(A.aZ1, m, n, face) + curl0_face(zcg, m, n, face)) + wobj;
        const double px = deltafnc_d(x, X, dx), py = deltafnc_d(y, Y, dx);
        gx += (dx * dx) * ddeltafnc_dr0(x, X, dx) * py * G;
        gy += (dx * dx) * px * ddeltafnc_dr0(y, Y, dx) * G;
      }
    }
    const double rx = X - C.pivot_x, ry = Y - C.pivot_y;
    const double dXdA = ry * sn, dYdA = -rx * sn;
    const double dVx = C.pitch_omega * cs * ry + thd * rx * sn;
    const double dVy = -C.pitch_omega * cs * rx + thd * ry * sn;
    part += gx * dXdA + gy * dYdA - dx * (A.aRf[k] * dVx + A.aRf[nb + k] * dVy);
  }
  __shared__ double red[128];
  red[threadIdx.x] = part;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *acc += red[0];
}

// Level-k CN adjoint, node part: r_hat = con1 A_hat + P_hat' ; P_hat = con2 A_hat
// (first step: rhs_old was set to rhs, so r_hat += con2 A_hat, P_hat = 0);
// ring part: lastbc_hat_k += vfac apply_bc^T(A_hat), ob_hat = vfac apply_bc^T(A_hat).
__global__ void k_adj_level(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids, int k, int first) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  if (k > C.L) return;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double del22 = C.delta * C.delta * (double)(1 << (2 * (k - 1)));
  double con1 = 1.5 * C.dt / del22 / C.norm, con2 = -0.5 * C.dt / del22 / C.norm;
  double vf = 0.5 * C.dt / C.re / del22 / C.norm;
  if (t < C.ns) {
    double ah = A.aA[t];
    double* P = A.aP + (size_t)(k - 1) * C.ns;
    double r = con1 * ah + P[t];
    if (first) { r += con2 * ah; P[t] = 0.0; }
    else P[t] = con2 * ah;
    A.aR[t] = r;
  } else if (t < C.ns + C.nring) {
    int r = t - C.ns;
    double v = vf * applybcT_at(A.aA, C.m, C.n, r);
    A.aLb[(size_t)(k - 1) * C.nring + r] += v;
    A.aObc[r] = v;
  }
}

// Transposed linearisation of nonlinear(omega, q, q0, bc) followed by rot,
// about the stored forward state (operators.f90:465-510, 291-304). With
// H = rot^T r_hat = curl(r_hat, 0):
//   node  omega_hat(i,j) += .5 va(i,j)(Hu(i,j-1)+Hu(i,j)) - .5 ua(i,j)(Hv(i-1,j)+Hv(i,j))
//   ring  lastbc_hat     += the same products at the edge entries
//   face  q_hat           = .5 * (adjoints of the face averages uavg / vavg)
__global__ void k_adj_nonlinear(const DevCase* __restrict__ cases, const AdjCase* __restrict__ adj, const int* __restrict__ cids, int k) {
  const int slot = blockIdx.z;
  const DevCase& C = cases[cids[slot]];
  const AdjCase& A = adj[slot];
  if (k > C.L) return;
  int m = C.m, n = C.n;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double* W = A.fwW + (size_t)(k - 1) * C.ns;
  const double* Q = A.fwQ + (size_t)(k - 1) * C.nq;
  const double* Q0 = C.q0 + (size_t)(k - 1) * C.nq;
  const double* Wc = k < C.L ? A.fwW + (size_t)k * C.ns : nullptr;  // level k+1, for lastbc
  const double* rh = A.aR;
  auto bcv = [&](int side, int I) { return Wc ? getbc_raw(Wc, m, n, side, I) * 0.25 : 0.0; };
  auto R = [&](int i, int j) { return rh[nidx(i, j, m)]; };
  // H = curl(r_hat, 0): u faces (i=2..m, j=1..n), v faces (i=1..m, j=2..n)
  auto Hu = [&](int i, int j) -> double {
    if (i < 2 || i > m || j < 1 || j > n) return 0.0;
    if (j == 1) return R(i, 2);
    if (j == n) return -R(i, n);
    return R(i, j + 1) - R(i, j);
  };
  auto Hv = [&](int i, int j) -> double {
    if (i < 1 || i > m || j < 2 || j > n) return 0.0;
    if (i == 1) return -R(2, j);
    if (i == m) return R(m, j);
    return R(i, j) - R(i + 1, j);
  };
  auto qt = [&](int face) { return Q[face] + Q0[face]; };
  auto va = [&](int i, int j) { return 0.5 * (qt(voff(i, j, m, n)) + qt(voff(i - 1, j, m, n))); };  // i=2..m
  auto ua = [&](int i, int j) { return 0.5 * (qt(uoff(i, j, m)) + qt(uoff(i, j - 1, m))); };      // j=2..n
  auto Wj = [&](int i, int j) -> double {  // omega extended along j (column i)
    if (j == 1) return bcv(SIDE_BOTTOM, i);
    if (j == n + 1) return bcv(SIDE_TOP, i);
    return W[nidx(i, j, m)];
  };
  auto Wi = [&](int i, int j) -> double {
    if (i == 1) return bcv(SIDE_LEFT, j);
    if (i == m + 1) return bcv(SIDE_RIGHT, j);
    return W[nidx(i, j, m)];
  };
  // adjoints of the averages
  auto vah = [&](int i, int j) { return 0.5 * Wj(i, j) * (Hu(i, j - 1) + Hu(i, j)); };   // i=2..m, j=1..n+1
  auto uah = [&](int i, int j) { return -0.5 * Wi(i, j) * (Hv(i - 1, j) + Hv(i, j)); };  // i=1..m+1, j=2..n
  if (t < C.ns) {
    int i = t % (m - 1) + 2, j = t / (m - 1) + 2;
    double v = 0.5 * va(i, j) * (Hu(i, j - 1) + Hu(i, j)) - 0.5 * ua(i, j) * (Hv(i - 1, j) + Hv(i, j));
    A.aW2[(size_t)(k - 1) * C.ns + t] += v;
  } else if (t < C.ns + C.nq) {
    int f = t - C.ns, nu = (m + 1) * n;
    double v = 0.0;
    if (f < nu) {  // u(i,j): uavg(i,j) [2<=j<=n] and uavg(i,j+1) [j+1<=n]
      int i = f % (m + 1) + 1, j = f / (m + 1) + 1;
      if (j >= 2) v += 0.5 * uah(i, j);
      if (j + 1 <= n) v += 0.5 * uah(i, j + 1);
    } else {  // v(i,j): vavg(i,j) [2<=i<=m] and vavg(i+1,j) [i+1<=m]
      int fv = f - nu, i = fv % m + 1, j = fv / m + 1;
      if (i >= 2) v += 0.5 * vah(i, j);
      if (i + 1 <= m) v += 0.5 * vah(i + 1, j);
    }
    A.aQ[(size_t)(k - 1) * C.nq + f] = v;
  } else if (t < C.ns + C.nq + C.nring) {
    int r = t - C.ns - C.nq;
    double v = 0.0;
    if (r < n + 1) { int J = r + 1; if (J >= 2 && J <= n) v = -0.5 * ua(1, J) * Hv(1, J); }
    else if (r < 2 * (n + 1)) { int J = r - (n + 1) + 1; if (J >= 2 && J <= n) v = -0.5 * ua(m + 1, J) * Hv(m, J); }
    else if (r < 2 * (n + 1) + m + 1) { int I = r - 2 * (n + 1) + 1; if (I >= 2 && I <= m) v = 0.5 * va(I, 1) * Hu(I, 1); }
    else { int I = r - 2 * (n + 1) - (m + 1) + 1; if (I >= 2 && I <= m) v = 0.5 * va(I, n + 1) * Hu(I, n); }
    A.aLb[(size_t)(k - 1) * C.nring + r] += v;
  }
}

// -------------------------------------------------------------------------
static dim3 grid_of(int count, int threads, const AdjGroup& g, int gy = 1) {
  return dim3((count + threads - 1) / threads, gy, g.n);
}
void adj_curlT(const AdjGroup& g, int nlev, int use_q1, cudaStream_t st) {
  k_adj_curlT<<<grid_of(g.max_ns + g.max_ring, 256, g, g.max_L), 256, 0, st>>>(g.dc, g.da, g.cids, nlev, use_q1);
}
void adj_v2f_level(const AdjGroup& g, int k, cudaStream_t st) {
  k_adj_v2f_level<<<grid_of(g.max_ns + g.max_ring, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, k);
}
void adj_getbcT(const AdjGroup& g, int which, int k, double fac, cudaStream_t st) {
  k_adj_getbcT<<<grid_of(g.max_perim, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, which, k, fac);
}
void adj_coarsifyT(const AdjGroup& g, int k, cudaStream_t st) {
  k_adj_coarsifyT<<<grid_of(g.max_ns, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, k);
  k_adj_zero_centre<<<grid_of(g.max_ns / 4 + 256, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, k);
}
void adj_force(const AdjGroup& g, cudaStream_t st) {
  k_adj_force<<<grid_of(g.max_nf, 128, g), 128, 0, st>>>(g.dc, g.da, g.cids);
}
void adj_solve(const AdjGroup& g, cudaStream_t st) {
  k_adj_tri<<<grid_of(g.max_nf, 8, g), 256, 0, st>>>(g.dc, g.da, g.cids, 0);
  k_adj_tri<<<grid_of(g.max_nf, 8, g), 256, 0, st>>>(g.dc, g.da, g.cids, 1);
}
void adj_rhsf(const AdjGroup& g, cudaStream_t st) {
  k_adj_rhsf<<<grid_of(std::max(g.max_nq, g.max_nf), 256, g), 256, 0, st>>>(g.dc, g.da, g.cids);
}
void adjm_reg_in(const AdjGroup& g, const double* const* xs, cudaStream_t st) {
  k_adjm_reg_in<<<grid_of(g.max_nq, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, xs);
}
void adjm_regT_curl0(const AdjGroup& g, double* const* outs, cudaStream_t st) {
  k_adjm_regT_curl0<<<grid_of(g.max_nf, 128, g), 128, 0, st>>>(g.dc, g.da, g.cids, outs);
}
void adjm_position(const AdjGroup& g, const AdjCase* acg, const double* const* us, double* accs, cudaStream_t st) {
  k_adjm_position<<<dim3(1, 1, g.n), 128, 0, st>>>(g.dc, g.da, g.cids, acg, us, accs);
}
void adj_level(const AdjGroup& g, int k, int first, cudaStream_t st) {
  k_adj_level<<<grid_of(g.max_ns + g.max_ring, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, k, first);
}
void adj_nonlinear(const AdjGroup& g, int k, cudaStream_t st) {
  k_adj_nonlinear<<<grid_of(g.max_ns + g.max_nq + g.max_ring, 256, g), 256, 0, st>>>(g.dc, g.da, g.cids, k);
}

}  // namespace ibfs
