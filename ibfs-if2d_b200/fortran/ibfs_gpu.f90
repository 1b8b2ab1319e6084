MODULE ibfs_gpu
  !---------------------------------------------------------------------------!
  ! iso_c_binding interface of the B200 IBFS time step (include/ibfs_capi.h).
  !
  ! The reference advances the flow with CALL advance(it) on module state
  ! (main.f90:47-50). With this module the Fortran host keeps its input,
  ! geometry and output code and hands the time step to the GPU library
  ! libibfs_b200.so: one handle per case, host arrays in the reference's own
  ! layouts (omega(2:m,2:n,mgridlev), q(Nq,mgridlev), fb(Nf), cholmat(Nf,Nf)).
  ! Every function returns an INTEGER(C_INT) status; ibfs_stop_on turns a
  ! failing status into STOP with the reference's message for that failure.
  !---------------------------------------------------------------------------!
  USE, INTRINSIC :: iso_c_binding
  IMPLICIT NONE

  INTEGER(C_INT), PARAMETER :: IBFS_OK = 0, IBFS_ERR_GRID = 1, IBFS_ERR_CHOL = 2, &
       IBFS_ERR_CG_MAXITER = 3, IBFS_ERR_CUDA = 4, IBFS_ERR_IO = 5, IBFS_ERR_TIMEOUT = 6, &
       IBFS_ERR_ARG = 7, IBFS_ERR_NOMEM = 8

  ! namelist READ_PARAMETERS, field for field (logicals as 0/1)
  TYPE, BIND(C) :: ibfs_params_c
     INTEGER(C_INT) :: istart, istop, isave
     INTEGER(C_INT) :: m, n
     REAL(C_DOUBLE) :: dt, re, cgtol
     INTEGER(C_INT) :: cg_max_iter
     INTEGER(C_INT) :: unif_flow
     REAL(C_DOUBLE) :: len, offsetx, offsety
     INTEGER(C_INT) :: mgridlev
     INTEGER(C_INT) :: make_vortex
     INTEGER(C_INT) :: stationary
  END TYPE ibfs_params_c

  ! options the reference fixes in source; all zero = reference behaviour
  TYPE, BIND(C) :: ibfs_options_c
     INTEGER(C_INT) :: precision, cg_relative, motion_kind
     REAL(C_DOUBLE) :: pitch_amp_deg, pitch_freq, pivot_x, pivot_y
     INTEGER(C_INT) :: tile_cfg
     INTEGER(C_INT) :: cg_precond
     INTEGER(C_INT) :: tc_tile
     INTEGER(C_INT) :: refine_slices
     INTEGER(C_INT) :: poisson_sweeps
  END TYPE ibfs_options_c

  INTERFACE
     INTEGER(C_INT) FUNCTION ibfs_create(p, opt, nb, xb, yb, bdyno, h) BIND(C, name="ibfs_create")
       IMPORT :: C_INT, C_DOUBLE, C_PTR, ibfs_params_c, ibfs_options_c
       TYPE(ibfs_params_c), INTENT(IN) :: p
       TYPE(ibfs_options_c), INTENT(IN) :: opt
       INTEGER(C_INT), VALUE :: nb
       REAL(C_DOUBLE), INTENT(IN) :: xb(*), yb(*)
       INTEGER(C_INT), INTENT(IN) :: bdyno(*)
       TYPE(C_PTR), INTENT(OUT) :: h
     END FUNCTION ibfs_create

     INTEGER(C_INT) FUNCTION ibfs_destroy(h) BIND(C, name="ibfs_destroy")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h
     END FUNCTION ibfs_destroy

     INTEGER(C_INT) FUNCTION ibfs_case_sizes(h, icase, m, n, nlev, nq, nb, nbody) &
          BIND(C, name="ibfs_case_sizes")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: icase
       INTEGER(C_INT), INTENT(OUT) :: m, n, nlev, nq, nb, nbody
     END FUNCTION ibfs_case_sizes

     INTEGER(C_INT) FUNCTION ibfs_set_state(h, icase, omega, fb, rhs_old, q, q0) BIND(C, name="ibfs_set_state")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: icase
       REAL(C_DOUBLE), INTENT(IN) :: omega(*), fb(*), rhs_old(*), q(*), q0(*)
     END FUNCTION ibfs_set_state

     INTEGER(C_INT) FUNCTION ibfs_get_state(h, icase, omega, fb, rhs_old, q, q0) BIND(C, name="ibfs_get_state")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: icase
       REAL(C_DOUBLE), INTENT(OUT) :: omega(*), fb(*), rhs_old(*), q(*), q0(*)
     END FUNCTION ibfs_get_state

     INTEGER(C_INT) FUNCTION ibfs_set_cholesky(h, icase, cholmat, cholvec) BIND(C, name="ibfs_set_cholesky")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: icase
       REAL(C_DOUBLE), INTENT(IN) :: cholmat(*), cholvec(*)
     END FUNCTION ibfs_set_cholesky

     INTEGER(C_INT) FUNCTION ibfs_get_cholesky(h, icase, cholmat, cholvec) BIND(C, name="ibfs_get_cholesky")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: icase
       REAL(C_DOUBLE), INTENT(OUT) :: cholmat(*), cholvec(*)
     END FUNCTION ibfs_get_cholesky

     INTEGER(C_INT) FUNCTION ibfs_precompute(h) BIND(C, name="ibfs_precompute")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h
     END FUNCTION ibfs_precompute

     ! body_vel may be C_NULL_PTR (no prescribed motion); fx, fy per body
     INTEGER(C_INT) FUNCTION ibfs_advance(h, itime, body_vel, fx, fy, circ, slip) BIND(C, name="ibfs_advance")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), INTENT(INOUT) :: itime
       TYPE(C_PTR), VALUE :: body_vel
       REAL(C_DOUBLE), INTENT(OUT) :: fx(*), fy(*), circ(*), slip
     END FUNCTION ibfs_advance

     INTEGER(C_INT) FUNCTION ibfs_advance_n(h, nsteps, hist) BIND(C, name="ibfs_advance_n")
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: nsteps
       TYPE(C_PTR), VALUE :: hist
     END FUNCTION ibfs_advance_n

     ! actuator jets on the last sum(npt) body points (actuation, grid.f90:579-633)
     INTEGER(C_INT) FUNCTION ibfs_set_actuators(h, icase, n_act, npt, u_j, u_j_osc, omg_j, theta_j) &
          BIND(C, name="ibfs_set_actuators")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       INTEGER(C_INT), VALUE :: icase, n_act
       INTEGER(C_INT), INTENT(IN) :: npt(*)
       REAL(C_DOUBLE), INTENT(IN) :: u_j(*), u_j_osc(*), omg_j(*), theta_j(*)
     END FUNCTION ibfs_set_actuators

     ! limit (seconds) of the split-precision GEMM's bounded device waits
     INTEGER(C_INT) FUNCTION ibfs_set_wait_limit(h, seconds, probe) BIND(C, name="ibfs_set_wait_limit")
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       TYPE(C_PTR), VALUE :: h
       REAL(C_DOUBLE), VALUE :: seconds
       INTEGER(C_INT), VALUE :: probe
     END FUNCTION ibfs_set_wait_limit

     TYPE(C_PTR) FUNCTION ibfs_last_error(h) BIND(C, name="ibfs_last_error")
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: h
     END FUNCTION ibfs_last_error
  END INTERFACE

CONTAINS

  FUNCTION ibfs_error_text(h) RESULT(msg)
    ! the library's message for the last failing call on h (or on no handle)
    TYPE(C_PTR), INTENT(IN) :: h
    CHARACTER(LEN=256) :: msg
    CHARACTER(KIND=C_CHAR), POINTER :: c(:)
    TYPE(C_PTR) :: p
    INTEGER :: i
    msg = ' '
    p = ibfs_last_error(h)
    IF (.NOT. C_ASSOCIATED(p)) RETURN
    CALL C_F_POINTER(p, c, [256])
    DO i = 1, 256
       IF (c(i) == C_NULL_CHAR) EXIT
       msg(i:i) = c(i)
    END DO
  END FUNCTION ibfs_error_text

  SUBROUTINE ibfs_stop_on(rc, h)
    ! A failing status ends the run the way the reference's own check does
    ! (grid.f90:68, operators.f90:784); the CG cap stays a warning
    ! (operators.f90:435-438).
    INTEGER(C_INT), INTENT(IN) :: rc
    TYPE(C_PTR), INTENT(IN) :: h
    SELECT CASE (rc)
    CASE (IBFS_OK)
       RETURN
    CASE (IBFS_ERR_CG_MAXITER)
       WRITE(111,*) "WARNING!! CJGR used max iterations!"
    CASE (IBFS_ERR_GRID)
       STOP 'HEY! Grid nodes must be divisible by 4!!'
    CASE (IBFS_ERR_CHOL)
       STOP 'choldc failed'
    CASE DEFAULT
       WRITE(*,*) 'IBFS GPU step failed: ', TRIM(ibfs_error_text(h))
       STOP 'ibfs_gpu: error'
    END SELECT
  END SUBROUTINE ibfs_stop_on

END MODULE ibfs_gpu
