/*
 * ibfs_capi.h -- C-ABI of the B200-native IBFS per-timestep advance.
 *
 * Drop-in seam for the reference's in-process call CALL advance(it)
 * (atchieu/ibfs-if2d src/main.f90:47-50) and its setup/output seams. Plain C
 * types only (no CUDA or torch types): callable from Fortran iso_c_binding,
 * C, C++ and ctypes. All arrays are host arrays in the reference's Fortran
 * column-major layouts, 1-based semantics as documented per entry point:
 *   omega, rhs_old  (m-1)*(n-1)*L   node (i,j), i=2..m fastest (variables.f90:46)
 *   q, q0           Nq*L            u(i,j)=i+(j-1)(m+1), v(i,j)=(m+1)n+i+(j-1)m
 *                                   (grid.f90:119-134), Nq=(m+1)n+(n+1)m
 *   fb, body_vel    Nf=2*Nb         x-components then y-components (grid.f90:105-116)
 *   cholmat, cholvec Nf*Nf, Nf      the ibfs.chd record (variables.f90:116-117)
 * Every entry point returns an int status (IBFS_OK = 0). Calls on one handle
 * are not reentrant; use one handle per host thread. Host arrays are never
 * retained past a call.
 */
#ifndef IBFS_CAPI_H
#define IBFS_CAPI_H

#ifdef __cplusplus
extern "C" {
#endif

#define IBFS_OK 0
#define IBFS_ERR_GRID 1        /* m or n not divisible by 4 (grid.f90:67-69)          */
#define IBFS_ERR_CHOL 2        /* non-positive pivot, 'choldc failed' (operators.f90:784) */
#define IBFS_ERR_CG_MAXITER 3  /* CG used cg_max_iter iterations (operators.f90:435-438);
                                  a warning, as in the reference: the step is complete and
                                  its outputs are returned                               */
#define IBFS_ERR_CUDA 4        /* CUDA runtime error; see ibfs_last_error              */
#define IBFS_ERR_IO 5          /* restart / Cholesky file read or write failed         */
#define IBFS_ERR_TIMEOUT 6     /* a bounded device wait gave up                        */
#define IBFS_ERR_ARG 7         /* invalid argument (null pointer, case index, size)    */
#define IBFS_ERR_NOMEM 8       /* device allocation failed                             */

/* Namelist READ_PARAMETERS, field for field (parameters.f90:12-31, 48-50).
 * Logical fields are ints (0 = .FALSE.). make_vortex is read but unused, as
 * in the reference. */
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
} ibfs_params_c;

/* Options that the reference fixes in source; zero-initialised = reference
 * behaviour, FP64. */
typedef struct {
  int precision;       /* 0: FP64 (plain method); 1: split-BF16 tensor-core transforms
                          with one FP64 refinement sweep per solve                        */
  int cg_relative;     /* 0: stop CG when r.r <= cgtol^2 (operators.f90:413-415);
                          1: stop when ||r|| <= cgtol*||b||                             */
  int motion_kind;     /* 0: body velocities from the caller per step (move_body,
                          grid.f90:523-576); 1: rigid pitching about (pivot_x,pivot_y),
                          alpha(t) = amp*sin(2 pi f t), points move, reg rebuilt        */
  double pitch_amp_deg, pitch_freq, pivot_x, pivot_y;
  int tile_cfg;        /* FP64 transform tile: 0..3 the unsplit shapes 64x64, 32x32,
                          64x32, 32x64 (bit-identical results); 4..6 split-K over a
                          cluster (32x32 in 2, 64x64 in 4, 32x32 in 4); -1 = the
                          measured autotuner                                        */
  int cg_precond;      /* CG cases: 0 = cjgr as in the reference (unpreconditioned);
                          1 = preconditioned CG: the force operator factored with the
                          body turned by the grid angle nearest the step's pitch
                          (A_k = L_k L_k^T, one slot per angle of a grid spacing at
                          most 1 degree, each factored like preprocess on first use),
                          applied as z = Q L_k^-T L_k^-1 Q^T r with Q the remaining
                          rotation of each point's (fx, fy); a body that does not move
                          has one slot. Same stop rule on the true residual        */
  int tc_tile;         /* split-precision form: tile configuration of the tensor-core
                          GEMM: 1 = 128x128 output tile, K blocks of 64, two pipeline
                          stages; 2 = 128x256, K blocks of 32, two stages; 3 = 128x128,
                          K blocks of 32, four stages; 4 = 256x256 on a pair of CTAs
                          (tcgen05 cta_group::2), K blocks of 64, two stages; 0 = the
                          measured autotuner picks per launch group. Taken from the
                          first case of a batch                                    */
  int refine_slices;   /* split-precision form: BF16 slices per operand in the correction
                          solves of the refinement: 0 = three (six products) for the
                          Poisson solves of vort2flux, two (three products) for the
                          well-conditioned Crank-Nicolson and ainv solves; 2 or 3 = that
                          many for all. Taken from the first case of a batch       */
  int poisson_sweeps;  /* split-precision form: FP64 residual-correction sweeps of the
                          Poisson (ctci) solves: 0 or 1 = one, 2 = two (each sweep
                          contracts their error by ~0.4 m^2 x 3e-7, ~0.03 at m = 512;
                          the other solves always get one). Taken from the first
                          case of a batch                                          */
} ibfs_options_c;

typedef struct ibfs_handle ibfs_handle;

/* setup + setup_variables with istart=0 (grid.f90:44-139, variables.f90:28-77):
 * grid indexing, level clamp (grid.f90:79-81), regularisation tables
 * (setup_reg, grid.f90:142-230), spectral tables (setup_fft, myfft.f90:21-70),
 * initial state (q0 = uniform flow when unif_flow). Body points as read from
 * geom.inp (grid.f90:270-277). opt may be NULL. */
int ibfs_create(const ibfs_params_c* p, const ibfs_options_c* opt, int nb, const double* xb,
                const double* yb, const int* bdyno, ibfs_handle** out);

/* Batched form: ncases independent cases of uneven sizes in one handle; one
 * launch per kernel serves all cases. p, opt, nb have ncases entries; xb, yb,
 * bdyno are the cases' body arrays concatenated. No reference counterpart
 * (the reference runs one case per process). */
int ibfs_batch_create(int ncases, const ibfs_params_c* p, const ibfs_options_c* opt, const int* nb,
                      const double* xb, const double* yb, const int* bdyno, ibfs_handle** out);

/* destroy_variables / destroy_grid (variables.f90:80-107). */
int ibfs_destroy(ibfs_handle* h);

/* Sizes after setup of case icase (mgridlev already clamped, grid.f90:81). */
int ibfs_case_sizes(const ibfs_handle* h, int icase, int* m, int* n, int* nlev, int* nq, int* nb,
                    int* nbody);
int ibfs_num_cases(const ibfs_handle* h);

/* read_variables / write_variables payload (variables.f90:141-175): the .var
 * record omega, fb, rhs_old, q, q0 in that order. Any pointer may be NULL. */
int ibfs_set_state(ibfs_handle* h, int icase, const double* omega, const double* fb,
                   const double* rhs_old, const double* q, const double* q0);
int ibfs_get_state(const ibfs_handle* h, int icase, double* omega, double* fb, double* rhs_old,
                   double* q, double* q0);

/* Vertex fields of one level for the Tecplot export (write_tecplot,
 * operators.f90:702-763, the post-processing step after the advance):
 * out[5][(m-1)*(n-1)], node (i,j) with i = 2..m fastest, the fields u, v,
 * etfx, etfy, vort in the reference's order and arithmetic (etf = reg(fb) on
 * the level-1 faces, del = 2^(level-1) delta). level is 1-based. */
int ibfs_vertex_fields(ibfs_handle* h, int icase, int level, double* out);

/* read_cholesky / write_cholesky payload (variables.f90:110-137): cholmat
 * (upper triangle = A, strict lower = factor) and cholvec (diagonal). */
int ibfs_set_cholesky(ibfs_handle* h, int icase, const double* cholmat, const double* cholvec);
int ibfs_get_cholesky(const ibfs_handle* h, int icase, double* cholmat, double* cholvec);

/* preprocess (operators.f90:29-59): A = [a_times(e_1) ... a_times(e_Nf)] built
 * as one multi-right-hand-side pass on the GPU, then choldc on the GPU. Runs
 * for every stationary case without a factor; ibfs_advance, ibfs_advance_n
 * and ibfs_batch_advance call it when a stationary case has none (the
 * reference's preprocess at itime == 1 reads input/ibfs.chd instead when that
 * file exists: give the factor with ibfs_set_cholesky before the first step).
 * Returns IBFS_ERR_CHOL on a non-positive pivot. */
int ibfs_precompute(ibfs_handle* h);

/* advance (operators.f90:62-188) of a single-case handle. *itime is
 * incremented as in the reference. body_vel: Nf body-point velocities in flow
 * units (NULL = none); scaled by delta as move_body does (grid.f90:573-574).
 * Outputs (any may be NULL): fx, fy per body (bodies minval..maxval(bdyno),
 * write_force operators.f90:583-659, already divided by dt and times 2*delta),
 * circ per level (write_circ :662-699), slip (write_slip :549-580). */
int ibfs_advance(ibfs_handle* h, int* itime, const double* body_vel, double* fx, double* fy,
                 double* circ, double* slip);

/* nsteps advances of every case, replayed from one captured CUDA graph per
 * step. hist (may be NULL) receives, per step, per case, the output block
 * [fx(nbody) fy(nbody) circ(L) slip]; ibfs_output_stride gives the doubles
 * of one step (all cases) and ibfs_output_offset a case's offset within it.
 * The body velocities are those of the last ibfs_advance/ibfs_batch_advance
 * (zero initially). */
int ibfs_advance_n(ibfs_handle* h, int nsteps, double* hist);

/* One advance of every case of a handle: the batched counterpart of
 * ibfs_advance (the reference runs one case per process, main.f90:42-54).
 * body_vel: every case's Nf body-point velocities in flow units, concatenated
 * in case order (NULL = 0); they stay in force for later ibfs_advance_n calls.
 * out (may be NULL): the step's outputs, ibfs_output_stride doubles laid out
 * as one step of ibfs_advance_n's history. */
int ibfs_batch_advance(ibfs_handle* h, const double* body_vel, double* out);
int ibfs_output_offset(const ibfs_handle* h, int icase);
int ibfs_output_stride(const ibfs_handle* h);

/* Individual operators of case 0 for verification (no reference counterpart
 * as an entry point; each applies one reference function):
 *   op 0 dst (myfft.f90:83-94)      in/out Ns
 *   op 1 ctci (myfft.f90:97-109)    in/out Ns
 *   op 2 ainv (myfft.f90:112-124)   in/out Ns
 *   op 3 a_times (operators.f90:444-462)  in/out Nf
 *   op 4 regT (operators.f90:531-546) in Nq, out Nf
 *   op 5 reg + rot (operators.f90:513-528, 291-304) in Nf, out Ns          */
int ibfs_apply_op(ibfs_handle* h, int op, const double* in, double* out);

/* Device timing of the last ibfs_advance_n call: total milliseconds. */
int ibfs_last_timing(const ibfs_handle* h, double* ms);

/* Number of kernel launches in one captured step graph (no reference
 * counterpart; reports the launch structure of the advance). */
int ibfs_kernels_per_step(const ibfs_handle* h);

/* Tile configurations (1..4, as ibfs_options_c.tc_tile) of the
 * split-precision form's tensor-core GEMM launch groups of the step program,
 * in launch order: writes up to max of them to cfgs (may be NULL) and
 * returns how many there are (0 for a plain FP64 handle). No reference
 * counterpart (reports the tuner's choice). */
int ibfs_gemm_tiles(const ibfs_handle* h, int* cfgs, int max);

/* Discrete adjoint of nsteps advances (no reference counterpart; the
 * reference has no derivatives). For a single-case handle, stationary body,
 * FP64 form: from the current state, with the body velocities body_vel (Nf,
 * flow units as in ibfs_advance, NULL = 0) held constant, it runs nsteps
 * advances and returns J = sum_s sum_b (wx[s*nbody+b] fx_b^s + wy[s*nbody+b]
 * fy_b^s) over the write_force outputs, and grad_vel = dJ/d body_vel (Nf).
 * Checkpoints of the state every checkpoint_every steps; each segment is
 * recomputed during the backward pass. The transposed operators: curl^T
 * (rot and ring terms), rot^T (curl with zero ring), get_bc^T, apply_bc^T,
 * coarsify^T, reg <-> regT, the linearised nonlinear term transposed; the DST
 * inverses and the Cholesky solve are self-adjoint. On return the state is
 * the state after the nsteps advances. ms_forward / ms_total (may be NULL):
 * device time of the forward pass and of the whole run. */
int ibfs_adjoint_run(ibfs_handle* h, int nsteps, int checkpoint_every, const double* body_vel, const double* wx,
                     const double* wy, double* J, double* grad_vel, double* ms_forward, double* ms_total);

/* Actuator jets (the reference's actuation, grid.f90:579-605, and u_jet,
 * :608-633): the last sum(npt) body points of case icase, npt[a] points per
 * actuator a = 0..n_act-1 in that order (the slot points actuator_slot
 * appends, grid.f90:636-718), get every step the velocity
 *   u_jet = (u_j + u_j_osc sin(omg_j dt itime)) (cos, sin)(pi/180 theta_j)
 * (flow units, multiplied by delta in the force system like the motion
 * vector), computed on the device after any body motion and overriding the
 * body velocities passed to ibfs_advance for those points. The parameters are
 * those of input/actuator.NNN.inp (&READ_ACT_PARAMETERS); the reference reads
 * them from the file every step. n_act = 0 removes the jets. Rebuilds the step
 * graph; call between advances. */
int ibfs_set_actuators(ibfs_handle* h, int icase, int n_act, const int* npt, const double* u_j,
                       const double* u_j_osc, const double* omg_j, const double* theta_j);

/* Discrete adjoint of nsteps advances of rigidly pitching bodies (no
 * reference counterpart): every case of the handle has motion_kind 1,
 * stationary = .FALSE. (CG force solve, cjgr operators.f90:393-441) and the
 * plain FP64 form, and all are at the same step. From the current states it
 * runs nsteps advances of the handle and returns, per case c,
 * J[c] = sum_s sum_b (wx[c][s][b] fx_b^s + wy[c][s][b] fy_b^s) and
 * dJ_damp[c] = dJ[c] / d(pitch_amp_deg of case c), per degree of amplitude;
 * wx and wy are case-major, nsteps x nbody(c) values per case. The cases are
 * differentiated together, one launch per stage for all of them. The
 * amplitude moves the body points (the regularisation weights of reg/regT,
 * setup_reg grid.f90:142-230, differentiated through the Roma-Peskin-Berger
 * kernel, grid.f90:233-249) and sets their velocities (the right-hand side of
 * the force system). The CG solve is differentiated as an exact solve: its
 * adjoint is a CG solve with the transposed force operator, stopped by the
 * same tolerance rule. Checkpoints every checkpoint_every steps as
 * ibfs_adjoint_run. On return the states are those after the nsteps
 * advances; ibfs_last_cg_iterations reports the largest adjoint CG iteration
 * count. Returns IBFS_ERR_CG_MAXITER (a warning, results valid) when a
 * forward or adjoint solve used cg_max_iter iterations. */
int ibfs_adjoint_pitch_run(ibfs_handle* h, int nsteps, int checkpoint_every, const double* wx, const double* wy,
                           double* J, double* dJ_damp, double* ms_forward, double* ms_total);

/* CG iterations of the last advance (largest over the handle's cases), as
 * cjgr reports them (operators.f90:439-440); 0 for Cholesky handles. */
int ibfs_last_cg_iterations(const ibfs_handle* h);

/* Advances one step without the graph, with CUDA events around every launch
 * on the handle's stream, and returns per launch class the summed device
 * milliseconds, the launch count and the algorithmic flops (arrays of 5):
 * 0 stencil / inter-level / IB, 1 FP64 transform GEMM, 2 tensor-core
 * transform GEMM, 3 force solve, 4 split/refinement. No reference
 * counterpart (measurement only). */
int ibfs_profile_step(ibfs_handle* h, double* ms, int* launches, double* flops);

/* 2-D DST-I (the reference's dst, myfft.f90:83-94) of a device field that
 * allocates no device memory. No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc where they need a transform -- a driver
 * whose memory pool owns all device memory, or a runtime that keeps the CUDA
 * allocator off its solver thread. d_in, d_out: device pointers to (m-1)*(n-1) doubles in the Fortran
 * node layout; stream: a cudaStream_t (NULL = default stream); the call is
 * asynchronous on it. Limit: m-1, n-1 <= 511 (grids up to 512x512 cells),
 * else IBFS_ERR_ARG. The intermediate product lives in one file-scope device
 * array of 511*511 doubles (2.09 MB per GPU that loads the library, kept
 * until exit), shared by all calls: calls that overlap on the GPU race and
 * must be serialised by the caller. The first call on a device looks up that
 * array's device address (with that device current); make the first call
 * before any stream capture. That address belongs to the device's primary
 * context (the CUDA runtime's) and is kept for the life of the process; it is
 * not looked up again after cudaDeviceReset. A CUDA error already pending on
 * the calling thread is left in place and the call returns IBFS_ERR_CUDA
 * without launching. Errors: ibfs_last_error(NULL). */
int ibfs_dst2d_noalloc(const double* d_in, double* d_out, int m, int n, void* stream);

/* Limit of every bounded device wait of the handle, in seconds (0..60; the
 * default is 1). The only device-side waits are the mbarrier waits of the
 * split-precision form's tensor-core GEMM; on a plain FP64 handle the call
 * has no effect. A wait that passes the limit makes its thread block stop
 * work, wait for its own copies and products still in flight, free its
 * tensor memory and return; the advance then returns IBFS_ERR_TIMEOUT with
 * the role, block and pipeline step of the first wait that gave up, and the
 * handle's state is undefined (destroy it). probe != 0 tests that path: every
 * thread block of the GEMM first waits on a barrier that nothing completes,
 * before it issues any copy or product, so each such wait gives up after
 * `seconds` and the next advance returns IBFS_ERR_TIMEOUT. The values are
 * read by the kernel from device memory, so they apply to captured step
 * graphs too. No reference counterpart (the reference has no device
 * waits). */
int ibfs_set_wait_limit(ibfs_handle* h, double seconds, int probe);

/* Message of the last error on this handle (or of the last failed create). */
const char* ibfs_last_error(const ibfs_handle* h);

#ifdef __cplusplus
}
#endif
#endif
