// ibfs_common.cuh -- device data layout and shared helpers of the B200 IBFS
// advance (the per-timestep path of atchieu/ibfs-if2d, src/operators.f90).
//
// HBM layout (per case, one arena): every field keeps the reference's Fortran
// column-major layout so state exchange is a plain copy:
//   omega, rhs_old, s : [L][(m-1)*(n-1)]   node (i,j), i=2..m fastest
//   q, q0             : [L][Nq]            u-faces u(i,j)=i+(j-1)(m+1), then
//                                          v-faces v(i,j)=(m+1)n+i+(j-1)m
//   fb, rhsf, motion  : [Nf]               x-forces then y-forces
//   lastbc            : [L][nring]         ring left|right|bottom|top
// Kernels are "grouped": they take a device array of items (case, level) so
// one launch serves one case (plain form) or many uneven cases (batched form).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ibfs {

struct DevCase {
  int m, n, L, ns, nq, nb, nf, nring;
  int nbody, bmin;
  double delta, dt, re, norm;
  // state
  double *omega, *rhs_old, *q, *q0, *fb;
  // q0 known in closed form: 1 when every level k holds q0_u1 * 2^(k-1) on
  // its u-faces and 0 on its v-faces (uniform flow, variables.f90:60-64, with
  // q0_u1 = delta; or no flow, q0_u1 = 0), so the stencils need not read it
  int q0_const;
  double q0_u1;
  // per-level work
  double *s;       // [L][ns] streamfunction per level
  double *lastbc;  // [L][nring]
  double *rhsA;    // [ns] combined right-hand side of the CN solve
  double *wa, *wb, *wc, *wd;  // [ns] transform scratch
  double *vort;    // [ns] scratch node field
  // spectral tables (cos(pi i/m), cos(pi j/n)) and sine matrices
  const double *cosx, *cosy;
  const double *Sm, *Sn;  // 2 sin(pi a b / m), (m-1)x(m-1) col-major
  // immersed boundary
  double *rhsf, *motion, *fwork, *bvel;     // [Nf]
  const int* face_ptr;  // [Nq+1] CSR by face: entries (force, weight) in reference k order
  const int* face_f;
  const double* face_w;
  const int* force_ptr;  // [Nf+1] CSR by force: entries (face, weight) by ascending face
  const int* force_face;
  const double* force_w;
  const double* wsum;    // [Nf] sum of a force's smear weights
  const int* bdyno;      // [Nb]
  double *Linv, *LinvT;  // [Nf*Nf] row-major inverse Cholesky factor and its transpose
  double* chol;          // [Nf*Nf] cholmat (Fortran layout) and cholvec after it
  // outputs of the last step
  double* out;  // fx[nbody], fy[nbody], circ[L], slip
  int* itime;   // device step counter
  int* status;  // device error flags

  // moving body (rigid pitching about a pivot): positions, and per-step
  // regularisation tables over a fixed patch of faces the body can reach
  int moving;
  double offx, offy;                                 // offsetx, offsety (grid origin)
  double pitch_amp, pitch_omega, pivot_x, pivot_y;  // amplitude (rad), 2 pi f
  const double *xb0, *yb0;  // positions at zero pitch
  double *xb, *yb;          // current positions
  int pu_i0, pu_j0, pu_w, pu_h;  // u-face patch: i in [pu_i0, pu_i0+pu_w), j in [pu_j0, pu_j0+pu_h)
  int pv_i0, pv_j0, pv_w, pv_h;  // v-face patch
  int* pcnt;                     // [patch faces] entries per face (u patch, then v patch)
  int* pf;                       // [patch faces][kPatchCap] force index, ascending body point
  double* pw;                    // [patch faces][kPatchCap] weight
  int* tcnt;                     // [Nf] faces per force (<= 9)
  int* tface;                    // [Nf][9] face index, ascending
  double* tw;                    // [Nf][9] weight
  double* twsum;                 // [Nf] sum of a force's weights
  double* tq;                    // [Nf][9] (q + q0) at the force's faces, or null (adjoint capture)

  // actuator jets (actuation / u_jet, grid.f90:579-633): the last nact body
  // points, [nact][5] = u_j, u_j_osc, omg_j, cos(pi/180 theta_j), sin(pi/180 theta_j)
  int nact;
  const double* act;

  // conjugate gradient (operators.f90:393-441) on the force system
  double *cg_r, *cg_d, *cg_q, *cg_q2;  // [Nf]
  double *cg_z, *cg_y;                 // [Nf] preconditioned residual and its half-solve (cg_pre)
  double* cg_sc;                       // delta_new (r.z), delta_old, eps, alpha, r.r
  int cg_pre;                          // preconditioned CG (factors of A at a grid of pitch angles)
  int pre_k0;                          // slot of zero pitch: slot k = body turned by (k - pre_k0) pre_dth
  double pre_dth;                      // pitch-angle grid spacing (radians)
  double* pre_fac;                     // [slots][2][Nf*Nf] Linv, LinvT of each slot (row-major)
  const int* pre_idx;                  // slot of the step being advanced (set by the host)
  int* cg_it;                          // iterations, active flag
  double cgtol;
  int cg_max_iter, cg_rel;
};

constexpr int kPatchCap = 12;

struct LevelItem {
  int c;  // case index
  int k;  // level, 1-based
};

// Fortran-style index helpers. Node arrays are declared DIMENSION(2:m,2:n):
__device__ __forceinline__ int nidx(int i, int j, int m) { return (i - 2) + (j - 2) * (m - 1); }
// assumed-shape sections (lower bound 1), used by get_bc/apply_bc:
__device__ __forceinline__ int ridx(int a, int b, int m) { return (a - 1) + (b - 1) * (m - 1); }
// 0-based face offsets of u(i,j), v(i,j):
__device__ __forceinline__ int uoff(int i, int j, int m) { return (i - 1) + (j - 1) * (m + 1); }
__device__ __forceinline__ int voff(int i, int j, int m, int n) { return (m + 1) * n + (i - 1) + (j - 1) * m; }

// Ring offsets (grid.f90:73-76).
__device__ __forceinline__ int ring_left(int, int) { return 0; }
__device__ __forceinline__ int ring_right(int, int n) { return n + 1; }
__device__ __forceinline__ int ring_bottom(int, int n) { return 2 * (n + 1); }
__device__ __forceinline__ int ring_top(int m, int n) { return 2 * (n + 1) + m + 1; }

enum Side { SIDE_LEFT = 0, SIDE_RIGHT = 1, SIDE_BOTTOM = 2, SIDE_TOP = 3 };

// get_bc (operators.f90:336-367) evaluated for one ring entry: the value the
// reference stores at rbc(side + I), I = 1..m+1 (bottom/top) or 1..n+1
// (left/right), before the final multiplication by fac. r is the coarser
// level's node field (assumed shape, 1-based).
__device__ __forceinline__ double getbc_raw(const double* __restrict__ r, int m, int n, int side, int I) {
  int t = I - 1;  // loop variable i (or j) of get_bc
  if (side == SIDE_BOTTOM || side == SIDE_TOP) {
    int b = (side == SIDE_BOTTOM) ? n / 4 : 3 * n / 4;
    if ((t & 1) == 0) return r[ridx(m / 4 + t / 2, b, m)];
    return 0.5 * (r[ridx(m / 4 + (t + 1) / 2, b, m)] + r[ridx(m / 4 - 1 + (t + 1) / 2, b, m)]);
  } else {
    int a = (side == SIDE_LEFT) ? m / 4 : 3 * m / 4;
    if ((t & 1) == 0) return r[ridx(a, n / 4 + t / 2, m)];
    return 0.5 * (r[ridx(a, n / 4 + (t + 1) / 2, m)] + r[ridx(a, n / 4 - 1 + (t + 1) / 2, m)]);
  }
}

__device__ __forceinline__ double ring_at(const double* __restrict__ ring, int m, int n, int side, int I) {
  int off = side == SIDE_LEFT ? 0 : side == SIDE_RIGHT ? n + 1 : side == SIDE_BOTTOM ? 2 * (n + 1) : 2 * (n + 1) + m + 1;
  return ring[off + I - 1];
}

// apply_bc (operators.f90:370-390) contribution to node r(a,b), added onto
// val in the reference's order: bottom/top loop first, then left/right.
// The ring value at side+I is supplied by a functor f(side, I).
template <class F>
__device__ __forceinline__ double apply_bc_at(double val, int a, int b, int m, int n, double fac, F f) {
  if (b == 1) val = val + fac * f(SIDE_BOTTOM, a + 1);
  if (b == n - 1) val = val + fac * f(SIDE_TOP, a + 1);
  if (a == 1) val = val + fac * f(SIDE_LEFT, b + 1);
  if (a == m - 1) val = val + fac * f(SIDE_RIGHT, b + 1);
  return val;
}

// lam(i,j) of myfft.f90:131-132 from the cosine tables.
__device__ __forceinline__ double lam_ij(double ci, double cj) { return -2.0 * (ci + cj - 2.0); }

// ---------------------------------------------------------------------------
// Immersed-boundary smearing shared by the advance and its adjoint.

// grid.f90:233-249.
__device__ __forceinline__ double deltafnc_d(double r, double r0, double dr) {
  double d = fabs(r - r0);
  if (d <= 0.5 * dr) {
    double t = (r - r0) / dr;
    return (1.0 + sqrt(-3.0 * t * t + 1.0)) / (3.0 * dr);
  } else if (d <= 1.5 * dr) {
    double a = fabs((r - r0) / dr);
    double u = 1.0 - a;
    return (5.0 - 3.0 * a - sqrt(-3.0 * u * u + 1.0)) / (6.0 * dr);
  }
  return 0.0;
}

// d/d r0 of deltafnc_d(r, r0, dr): with t = (r - r0)/dr and deltafnc = psi(t)/dr,
// psi'(t) = -t / sqrt(1 - 3t^2) on |t| <= 1/2 and
// -sgn(t) (1 + (1-|t|) / sqrt(1 - 3(1-|t|)^2)) / 2 on 1/2 < |t| <= 3/2
// (continuous at both joins, zero at |t| = 3/2), so d/dr0 = -psi'(t) / dr^2.
__device__ __forceinline__ double ddeltafnc_dr0(double r, double r0, double dr) {
  double d = fabs(r - r0);
  double t = (r - r0) / dr;
  double dpsi;
  if (d <= 0.5 * dr) {
    dpsi = -t / sqrt(-3.0 * t * t + 1.0);
  } else if (d <= 1.5 * dr) {
    double u = 1.0 - fabs(t);
    dpsi = -copysign(1.0, t) * 0.5 * (1.0 + u / sqrt(-3.0 * u * u + 1.0));
  } else {
    return 0.0;
  }
  return -dpsi / (dr * dr);
}

// reg (operators.f90:513-528) at one face: stationary bodies gather from the
// CSR-by-face table whose entries keep the reference's smear order; moving
// bodies from the patch tables rebuilt every step.
__device__ __forceinline__ double reg_face(const DevCase& C, const double* __restrict__ f, int face) {
  if (C.moving) {  // patch tables rebuilt every step
    int m = C.m, nu = (m + 1) * C.n, pidx;
    if (face < nu) {
      int i = face % (m + 1) + 1 - C.pu_i0, j = face / (m + 1) + 1 - C.pu_j0;
      if (i < 0 || j < 0 || i >= C.pu_w || j >= C.pu_h) return 0.0;
      pidx = i + j * C.pu_w;
    } else {
      int fv = face - nu;
      int i = fv % m + 1 - C.pv_i0, j = fv / m + 1 - C.pv_j0;
      if (i < 0 || j < 0 || i >= C.pv_w || j >= C.pv_h) return 0.0;
      pidx = C.pu_w * C.pu_h + i + j * C.pv_w;
    }
    double h = 0.0;
    for (int p = 0; p < C.pcnt[pidx]; p++) h = h + C.pw[pidx * kPatchCap + p] * f[C.pf[pidx * kPatchCap + p]];
    return h;
  }
  int p0 = C.face_ptr[face], p1 = C.face_ptr[face + 1];
  double h = 0.0;
  for (int p = p0; p < p1; p++) h = h + C.face_w[p] * f[C.face_f[p]];
  return h;
}

// regT (operators.f90:531-546) for one force: its faces in ascending order.
__device__ __forceinline__ double regT_force(const DevCase& C, const double* __restrict__ h, int f) {
  if (C.moving) {
    double s = 0.0;
    for (int p = 0; p < C.tcnt[f]; p++) s = s + C.tw[f * 9 + p] * h[C.tface[f * 9 + p]];
    return s;
  }
  int p0 = C.force_ptr[f], p1 = C.force_ptr[f + 1];
  double s = 0.0;
  for (int p = p0; p < p1; p++) s = s + C.force_w[p] * h[C.force_face[p]];
  return s;
}

}  // namespace ibfs

#define IBFS_CUDA_CHECK(x)                                  \
  do {                                                      \
    cudaError_t e_ = (x);                                   \
    if (e_ != cudaSuccess) return ::ibfs::fail_cuda(e_, #x); \
  } while (0)
