// ibfs_adjoint.cuh -- buffers and launchers of the discrete adjoint.
#pragma once
#include "ibfs_common.cuh"

namespace ibfs {

// Adjoint working set of one case. "Hat" quantities are adjoints (dJ/dx).
struct AdjCase {
  double *aW, *aW2;  // [L][ns] adjoint of omega: incoming/in progress, and of the step-start omega
  double* aP;        // [L][ns] adjoint of rhs_old
  double* aQ;        // [L][nq] adjoint of q
  double* aQ1;       // [nq]    adjoint of the level-1 flux formed for the force solve
  double* aS;        // [L][ns] adjoint of the streamfunction
  double* aSbc;      // [L][nring] adjoint of its boundary ring
  double* aLb;       // [L][nring] adjoint of lastbc
  double* aObc;      // [nring] adjoint of omega_bc of the level being processed
  double *aA, *aZ1, *aZ2, *aR, *aT1, *aT2;  // [ns] node scratch
  double *aF, *aRf, *aTmp;                  // [nf] force-space scratch
  double* aGrad;     // [nf] dJ / d(body velocity)
  const double* fwW; // forward omega at the start of the step being differentiated
  const double* fwQ; // forward q at the start of that step
  const double* wx;  // [nbody] objective weights of the step's forces
  const double* wy;
  const double* tq;  // [nf][9] (q1 + q0) at each force's faces in that step (moving body)
};

// The slots of one adjoint program: slot i differentiates case cids[i] of the
// handle's device case array dc with working set da[i]; the maxima size the
// grids (max_perim: nodes on the get_bc box perimeter).
struct AdjGroup {
  int n = 0;
  const int* cids = nullptr;
  const DevCase* dc = nullptr;
  const AdjCase* da = nullptr;
  int max_ns = 0, max_nq = 0, max_nf = 0, max_ring = 0, max_L = 0, max_perim = 0;
};

enum { GETBC_SBC = 0, GETBC_OBC = 1, GETBC_LB = 2 };

void adj_curlT(const AdjGroup& g, int nlev, int use_q1, cudaStream_t st);
void adj_v2f_level(const AdjGroup& g, int k, cudaStream_t st);
void adj_getbcT(const AdjGroup& g, int which, int k, double fac, cudaStream_t st);
void adj_coarsifyT(const AdjGroup& g, int k, cudaStream_t st);
void adj_force(const AdjGroup& g, cudaStream_t st);
void adj_solve(const AdjGroup& g, cudaStream_t st);
void adj_rhsf(const AdjGroup& g, cudaStream_t st);
void adjm_reg_in(const AdjGroup& g, const double* const* xs, cudaStream_t st);
void adjm_regT_curl0(const AdjGroup& g, double* const* outs, cudaStream_t st);
void adjm_position(const AdjGroup& g, const AdjCase* acg, const double* const* us, double* accs, cudaStream_t st);
void adj_level(const AdjGroup& g, int k, int first, cudaStream_t st);
void adj_nonlinear(const AdjGroup& g, int k, cudaStream_t st);

}  // namespace ibfs
