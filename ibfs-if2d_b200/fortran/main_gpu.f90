PROGRAM main_gpu
  !---------------------------------------------------------------------------!
  ! The reference's main program (main.f90:12-63) with the time step on the
  ! GPU. Compiled together with the reference's own modules parameters, grid,
  ! variables and operators (all of src/ except main.f90), the module ibfs_gpu
  ! of this directory, and linked with libibfs_b200.so. Input, geometry,
  ! restart and Cholesky files and the force/circ/slip histories keep the
  ! reference's names and layouts; only CALL advance(it) is replaced.
  !---------------------------------------------------------------------------!
  USE, INTRINSIC :: iso_c_binding
  USE parameters
  USE grid
  USE variables
  USE ibfs_gpu

  IMPLICIT NONE
  TYPE(ibfs_params_c) :: p
  TYPE(ibfs_options_c) :: opt
  TYPE(C_PTR) :: h
  INTEGER(C_INT) :: rc, itime, gm, gn, glev, gnq, gnb, gnbody
  REAL(C_DOUBLE), ALLOCATABLE :: fx(:), fy(:), circ(:)
  REAL(C_DOUBLE) :: slip
  LOGICAL :: readchol

  OPEN(unit=111,file='output/ibfs.inf',status='unknown',position='append',form='formatted')
  WRITE(111,*) "==================================="
  WRITE(111,*) "|   Welcome to IBFS MGRID v1.0    |"
  WRITE(111,*) "|   (time step on the GPU)        |"
  WRITE(111,*) "==================================="

  ! SETUP SIMULATION: the reference's own input, grid and variables
  CALL input
  CALL setup
  CALL setup_variables

  ! THE GPU CASE: same parameters, same body points, same initial state
  p = ibfs_params_c(istart, istop, isave, m, n, dt, Re, cgtol, cg_max_iter, MERGE(1, 0, unif_flow), &
                    len, offsetx, offsety, mgridlev, MERGE(1, 0, make_vortex), MERGE(1, 0, stationary))
  opt = ibfs_options_c(0, 0, 0, 0.d0, 0.d0, 0.d0, 0.d0, -1)
  rc = ibfs_create(p, opt, INT(nb, C_INT), xb, yb, INT(bdyno, C_INT), h)
  CALL ibfs_stop_on(rc, h)
  rc = ibfs_case_sizes(h, 0_C_INT, gm, gn, glev, gnq, gnb, gnbody)
  ALLOCATE( fx(MAX(gnbody,1)), fy(MAX(gnbody,1)), circ(glev) )
  rc = ibfs_set_state(h, 0_C_INT, omega, fb, rhs_old, q, q0)
  CALL ibfs_stop_on(rc, h)
  IF (istart > 0 .AND. stationary) THEN   ! factor read by setup_variables
     rc = ibfs_set_cholesky(h, 0_C_INT, cholmat, cholvec)
     CALL ibfs_stop_on(rc, h)
  END IF

  ! BEGIN TIME MARCH
  itime = istart
  DO WHILE (itime < istop)
     IF (itime == 0 .AND. stationary) THEN  ! preprocess (operators.f90:29-59)
        INQUIRE(file='input/ibfs.chd',exist=readchol)
        IF (readchol) THEN
           CALL read_cholesky
           rc = ibfs_set_cholesky(h, 0_C_INT, cholmat, cholvec)
        ELSE
           rc = ibfs_precompute(h)
           CALL ibfs_stop_on(rc, h)
           rc = ibfs_get_cholesky(h, 0_C_INT, cholmat, cholvec)
           CALL write_cholesky
        END IF
        CALL ibfs_stop_on(rc, h)
     END IF
     WRITE(*,*) "* For itime =", itime + 1
     WRITE(111,*) "...Advancing to itime =", itime + 1
     rc = ibfs_advance(h, itime, C_NULL_PTR, fx, fy, circ, slip)
     CALL ibfs_stop_on(rc, h)

     IF ((MOD(itime,isave).EQ.0).OR.(itime==istop)) THEN
        rc = ibfs_get_state(h, 0_C_INT, omega, fb, rhs_old, q, q0)
        CALL write_variables(itime)
     END IF
     CALL append_history('output/force.dat', itime, [fx(1:gnbody), fy(1:gnbody)])
     CALL append_history('output/circ.dat', itime, circ)
     CALL append_history('output/slip.dat', itime, [slip])
     WRITE(*,*) "SLIP =", slip
  END DO

  rc = ibfs_destroy(h)
  CALL destroy_variables
  CALL destroy_grid
  CALL CPU_TIME(cputime)
  WRITE(*,*) "Total run time: ",cputime," s"
  WRITE(111,*) "Total run time: ",cputime," s"

CONTAINS

  SUBROUTINE append_history(fname, it, vals)
    ! write_force / write_circ / write_slip file handling (operators.f90:564-573)
    CHARACTER(*), INTENT(IN) :: fname
    INTEGER(C_INT), INTENT(IN) :: it
    REAL(C_DOUBLE), INTENT(IN) :: vals(:)
    LOGICAL :: ex
    INTEGER :: k
    INQUIRE(file=fname, exist=ex)
    IF (it == 1 .OR. .NOT. ex) THEN
       OPEN(unit=100, file=fname, form="formatted", status="replace")
    ELSE
       OPEN(unit=100, file=fname, form="formatted", status="old", position="append")
    END IF
    WRITE(100,*) it, (vals(k), k=1,SIZE(vals))
    CLOSE(100)
  END SUBROUTINE append_history

END PROGRAM main_gpu
