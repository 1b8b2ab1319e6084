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

void adj_curlT(const DevCase* c, const AdjCase* a, const DevCase& h, int nlev, int use_q1, cudaStream_t st);
void adj_v2f_level(const DevCase* c, const AdjCase* a, const DevCase& h, int k, cudaStream_t st);
void adj_getbcT(const DevCase* c, const double* ring, double* dst, const DevCase& h, double fac, cudaStream_t st);
void adj_coarsifyT(const DevCase* c, const AdjCase* a, const DevCase& h, int k, cudaStream_t st);
void adj_force(const DevCase* c, const AdjCase* a, const DevCase& h, cudaStream_t st);
void adj_solve(const DevCase* c, const double* in, double* tmp, double* out, const DevCase& h, cudaStream_t st);
void adj_rhsf(const DevCase* c, const AdjCase* a, const DevCase& h, cudaStream_t st);
void adj_level(const DevCase* c, const AdjCase* a, const DevCase& h, int k, int first, cudaStream_t st);
void adjm_reg_in(const DevCase* c, const AdjCase* a, const double* x, const DevCase& h, cudaStream_t st);
void adjm_regT_curl0(const DevCase* c, const AdjCase* a, double* out, const DevCase& h, cudaStream_t st);
void adjm_position(const DevCase* c, const AdjCase* a, const double* zcg, const double* u, double* acc,
                   cudaStream_t st);
void adj_nonlinear(const DevCase* c, const AdjCase* a, const DevCase& h, int k, cudaStream_t st);

}  // namespace ibfs
