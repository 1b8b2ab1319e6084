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
  opt = ibfs_options_c(0, 0, 0, 0.d0, 0.d0, 0.d0, 0.d0, -1, 0)
  rc = ibfs_create(p, opt, INT(nb, C_INT), xb, yb, INT(bdyno, C_INT), h)
  CALL ibfs_stop_on(rc, h)
  rc = ibfs_case_sizes(h, 0_C_INT, gm, gn, glev, gnq, gnb, gnbody)
  ALLOCATE( fx(MAX(gnbody,1)), fy(MAX(gnbody,1)), circ(glev) )
  rc = ibfs_set_state(h, 0_C_INT, omega, fb, rhs_old, q, q0)
  CALL ibfs_stop_on(rc, h)
  ! ACTUATOR JETS (actuation, grid.f90:579-633): setup counted n_act; the jets
  ! run on the device with each actuator's namelist read once
  IF (n_act > 0) CALL set_jets(n_act)
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

  SUBROUTINE set_jets(na)
    ! the parameters u_jet reads (grid.f90:616-623) and the point counts
    ! actuation reads (grid.f90:592-595), for actuators 1..na in order
    INTEGER, INTENT(IN) :: na
    INTEGER(C_INT) :: npt(na), rcj
    REAL(C_DOUBLE) :: uj(na), uosc(na), omg(na), th(na)
    REAL(KIND(0.D0)) :: x_j, y_j, h_j, u_j, u_j_osc, theta_j, omg_j
    NAMELIST /read_act_parameters/ x_j, y_j, h_j, u_j, u_j_osc, theta_j, omg_j
    CHARACTER(3) :: act_num
    INTEGER :: i
    DO i = 1, na
       WRITE(act_num,"(I3.3)") i
       x_j = 0.d0; y_j = 0.d0; h_j = 0.d0; u_j = 0.d0; u_j_osc = 0.d0; theta_j = 0.d0; omg_j = 0.d0
       OPEN(unit=7, file="input/actuator."//act_num//".inp", form="formatted", status="old")
       READ(unit=7, nml=read_act_parameters)
       CLOSE(7)
       OPEN(unit=7, file="input/slot."//act_num//".inp", form="formatted", status="old")
       READ(7,*) npt(i)
       CLOSE(7)
       uj(i) = u_j; uosc(i) = u_j_osc; omg(i) = omg_j; th(i) = theta_j
    END DO
    rcj = ibfs_set_actuators(h, 0_C_INT, INT(na, C_INT), npt, uj, uosc, omg, th)
    CALL ibfs_stop_on(rcj, h)
  END SUBROUTINE set_jets

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
