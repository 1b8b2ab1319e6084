/*
 * ibfs_oracle.h -- CPU FP64 restatement of the IBFS per-timestep advance.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
 * load it. The product path (ibfs-if2d_b200/) never links or calls it.
 *
 * It restates, loop by loop, the reference Fortran (atchieu/ibfs-if2d):
 *   src/operators.f90  advance / vort2flux / curl / rot / coarsify / get_bc /
 *                      apply_bc / cjgr / a_times / nonlinear / reg / regT /
 *                      write_force / write_circ / write_slip / choldc / cholsl
 *   src/myfft.f90      setup_fft tables, dst / ctci / ainv
 *   src/grid.f90       setup (indexing, level clamp), setup_reg, deltafnc
 *   src/variables.f90  setup_variables (initial state)
 * Each function below names the file:line it follows.
 *
 * The 2-D DST-I (FFTW RODFT00 in the reference, myfft.f90:115) is computed
 * with this file's own mixed-radix FFT of the odd extension (length 2m).
 *
 * Parity status: the reference Fortran+FFTW binary cannot be built here (no
 * Fortran compiler, no FFTW). The DST is pinned against scipy.fft.dst(type=1)
 * (same definition as RODFT00) and the whole advance is cross-checked against
 * an independent numpy restatement (tests/golden/make_golden.py). Parity with
 * the Fortran binary itself is therefore UNPINNED.
 *
 * Arrays use the reference's Fortran column-major layouts:
 *   omega, rhs_old: (m-1) x (n-1) x L, x fastest           (variables.f90:46)
 *   q, q0:          Nq x L, u-faces then v-faces           (grid.f90:119-134)
 *   fb:             Nf = 2 Nb, x-forces then y-forces      (grid.f90:105-116)
 *   bc ring:        2(m+1)+2(n+1), left|right|bottom|top    (grid.f90:73-76)
 */
#ifndef IBFS_ORACLE_H
#define IBFS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* The 16 fields of namelist READ_PARAMETERS (parameters.f90:48-50). */
typedef struct {
  int istart, istop, isave;
  int m, n;
  double dt, re, cgtol;
  int cg_max_iter;
  int unif_flow;
  double len, offsetx, offsety;
  int mgridlev;
  int make_vortex;
  int stationary;
} or_params;

typedef struct or_case or_case;

/* setup (grid.f90:44-139) + setup_variables (variables.f90:28-77) with
 * istart=0. Returns 0, or 1 if m,n not divisible by 4 (grid.f90:67-69). */
int or_create(const or_params* p, int nb, const double* xb, const double* yb,
              const int* bdyno, or_case** out);
void or_destroy(or_case* c);

/* Sizes after setup (mgridlev already clamped, grid.f90:79-81). */
void or_sizes(const or_case* c, int* m, int* n, int* nlev, int* nq, int* nb,
              int* nsmear, double* delta);

/* State exchange, same order/shape as the .var record (variables.f90:152). */
void or_get_state(const or_case* c, double* omega, double* fb, double* rhs_old,
                  double* q, double* q0);
void or_set_state(or_case* c, const double* omega, const double* fb,
                  const double* rhs_old, const double* q, const double* q0);
void or_get_cholesky(const or_case* c, double* cholmat, double* cholvec);
void or_set_cholesky(or_case* c, const double* cholmat, const double* cholvec);

/* Move body points and rebuild the smearing tables (setup_reg). */
void or_set_body(or_case* c, const double* xb, const double* yb);

/* preprocess: build A column by column and factor it (operators.f90:29-59).
 * Returns 0, or 2 if choldc meets a non-positive pivot (operators.f90:784). */
int or_preprocess(or_case* c);

/* advance (operators.f90:62-188). itime is incremented as in the reference.
 * body_vel: Nf prescribed body-point velocities (x then y) in flow units, or
 * NULL for none; they are scaled by delta as move_body does (grid.f90:573).
 * Outputs (any may be NULL): fx, fy per body (bodies minval..maxval of bdyno),
 * circ per level, slip, cg iterations. Returns 0, 2 (Cholesky failure) or
 * 3 (CG hit cg_max_iter). cg_rel != 0 makes CG stop on ||r|| <= cgtol*||b||. */
int or_advance(or_case* c, int* itime, const double* body_vel, double* fx,
               double* fy, double* circ, double* slip, int* cg_iters);
void or_set_cg_relative(or_case* c, int cg_rel);

/* Individual operators (for unit tests). Node arrays are (m-1)x(n-1). */
void or_dst(or_case* c, const double* in, double* out);
void or_ctci(or_case* c, const double* in, double* out);
void or_ainv(or_case* c, const double* in, double* out);
void or_curl(const or_case* c, const double* x, const double* xbc, double* out);
void or_rot(const or_case* c, const double* x, double* out);
void or_nonlinear(const or_case* c, const double* omega, const double* q,
                  const double* q0, const double* bc, double* fq);
void or_coarsify(const or_case* c, const double* crhs, const double* rhs,
                 double* out);
void or_get_bc(const or_case* c, const double* r, double* rbc, double fac);
void or_apply_bc(const or_case* c, double* r, const double* rbc, double fac);
void or_reg(const or_case* c, const double* h0, double* h);
void or_regT(const or_case* c, const double* h, double* h0);
void or_vort2flux(or_case* c, double* vel, double* omega, int nlev);
void or_a_times(or_case* c, const double* x, double* out);
void or_cholsl(const or_case* c, const double* b, double* x);
void or_tables(const or_case* c, double* lam, double* laminv, double* lam1,
               double* lam1i, double* con1, double* con2, double* vfac);
double or_deltafnc(double r, double r0, double dr);
int or_nlevmax(int m, int n);

#ifdef __cplusplus
}
#endif
#endif
