! ow3d_iface.f90 -- Fortran 2003 (iso_c_binding) interface to the C ABI of
! include/ow3d.h, for the reference program to call the B200 path.
!
! Add this file to the reference's src/ and link with -L<dir> -low3d -lcudart.
! No Fortran compiler exists where this library is built, so this module is
! not compile-checked there; tests/test_capi.py checks that the opaque
! parameter block below has the size of the C struct ow3d_params.
!
! Two ways to use it (one per boundary):
!
! (a) Replace only the Laplace solve. The four call sites of
!     src/timeintegration/Runge_Kutta_4.f90 pass the surface that defines the
!     sigma coefficients of that solve (DetermineTransformationConstantsArray
!     is called with the same structure just before each):
!       stages 1-3 (:129, :216, :309) solve on the stage surface
!         ierr = ow3d_solve(ow3d_h, RHS, PHI, Wavefield_tmp%E, Wavefield_tmp%Ex, &
!                           Wavefield_tmp%Exx, Wavefield_tmp%Ey, Wavefield_tmp%Eyy, iters)
!       the 4th solve (:419) is at the new time level
!         ierr = ow3d_solve(ow3d_h, RHS, PHI, Wavefield%E, Wavefield%Ex, &
!                           Wavefield%Exx, Wavefield%Ey, Wavefield%Eyy, iters)
!     in place of
!         CALL iterative_solution(RHS, n_rows, BuildLinearSystem, PHI, FineGrid)
!     ierr = OW3D_NOT_CONVERGED is the reference's silent non-convergence
!     (iterative_solution.f90:117-134): a warning; ierr < 0 is an error.
!
! (b) Replace the whole time step: ow3d_set_state once after set-up, then
!     ierr = ow3d_step(ow3d_h, 1) in place of CALL timeintegration_fsbc
!     (src/main/OceanWave3DTakeATimeStep.f90:27), ow3d_get_state whenever the
!     host needs E, P, W or PHI.
MODULE ow3d_iface
  USE, INTRINSIC :: iso_c_binding
  IMPLICIT NONE
  INTEGER(c_int), PARAMETER :: OW3D_OK = 0, OW3D_NOT_CONVERGED = 1
  INTEGER(c_int), PARAMETER :: OW3D_ERR_BAD_INPUT = -1, OW3D_ERR_CUDA = -2, OW3D_ERR_OOM = -3
  INTEGER(c_int), PARAMETER :: OW3D_ERR_UNSTABLE = -4, OW3D_ERR_TIMEOUT = -5, OW3D_ERR_NO_DEVICE = -6
  INTEGER(c_int), PARAMETER :: OW3D_ERR_IO = -7, OW3D_ERR_UNSUPPORTED = -8
  INTEGER(c_int), PARAMETER :: OW3D_SMOOTHER_MULTICOLOUR = 0, OW3D_SMOOTHER_LEXICOGRAPHIC = 1

  ! ow3d_params mirrors the deck (include/ow3d.h); filled by ow3d_read_deck
  ! and opaque to Fortran
  TYPE, BIND(C) :: ow3d_params_t
     INTEGER(c_int8_t) :: raw(2480)         ! opaque to Fortran: sizeof(ow3d_params)
  END TYPE

  INTERFACE
     INTEGER(c_int) FUNCTION ow3d_read_deck(path, p) BIND(C, name="ow3d_read_deck")
       IMPORT :: c_int, c_char, ow3d_params_t
       CHARACTER(kind=c_char), DIMENSION(*), INTENT(IN) :: path   ! NUL-terminated
       TYPE(ow3d_params_t), INTENT(OUT) :: p
     END FUNCTION

     INTEGER(c_int) FUNCTION ow3d_create(p, h, hx, hxx, hy, hyy, handle) BIND(C, name="ow3d_create")
       IMPORT :: c_int, c_double, c_ptr, ow3d_params_t
       TYPE(ow3d_params_t), INTENT(IN) :: p
       REAL(c_double), DIMENSION(*), INTENT(IN) :: h, hx, hxx, hy, hyy
       TYPE(c_ptr), INTENT(OUT) :: handle
     END FUNCTION

     INTEGER(c_int) FUNCTION ow3d_destroy(handle) BIND(C, name="ow3d_destroy")
       IMPORT :: c_int, c_ptr
       TYPE(c_ptr), VALUE :: handle
     END FUNCTION

     ! replaces CALL iterative_solution(RHS, N, BuildLinearSystem, PHI, FineGrid)
     INTEGER(c_int) FUNCTION ow3d_solve(handle, rhs, phi, E, Ex, Exx, Ey, Eyy, iters) BIND(C, name="ow3d_solve")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       REAL(c_double), DIMENSION(*), INTENT(IN) :: rhs
       REAL(c_double), DIMENSION(*), INTENT(INOUT) :: phi
       REAL(c_double), DIMENSION(*), INTENT(IN) :: E, Ex, Exx, Ey, Eyy
       INTEGER(c_int), INTENT(OUT) :: iters
     END FUNCTION

     ! y = A(eta) phi with the high-order operator (BuildLinearSystem)
     INTEGER(c_int) FUNCTION ow3d_matvec(handle, phi, y, E, Ex, Exx, Ey, Eyy) BIND(C, name="ow3d_matvec")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       REAL(c_double), DIMENSION(*), INTENT(IN) :: phi
       REAL(c_double), DIMENSION(*), INTENT(OUT) :: y
       REAL(c_double), DIMENSION(*), INTENT(IN) :: E, Ex, Exx, Ey, Eyy
     END FUNCTION

     INTEGER(c_int) FUNCTION ow3d_set_state(handle, E, P, W, phi, t) BIND(C, name="ow3d_set_state")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       REAL(c_double), DIMENSION(*), INTENT(IN) :: E, P, W, phi
       REAL(c_double), VALUE :: t
     END FUNCTION

     INTEGER(c_int) FUNCTION ow3d_put_surface(handle, E, P) BIND(C, name="ow3d_put_surface")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       REAL(c_double), DIMENSION(*), INTENT(IN) :: E, P
     END FUNCTION

     ! replaces CALL timeintegration_fsbc (nsteps = 1 per call)
     INTEGER(c_int) FUNCTION ow3d_step(handle, nsteps) BIND(C, name="ow3d_step")
       IMPORT :: c_int, c_ptr
       TYPE(c_ptr), VALUE :: handle
       INTEGER(c_int), VALUE :: nsteps
     END FUNCTION

     INTEGER(c_int) FUNCTION ow3d_get_state(handle, E, P, W, phi, t) BIND(C, name="ow3d_get_state")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       REAL(c_double), DIMENSION(*), INTENT(OUT) :: E, P, W, phi
       REAL(c_double), INTENT(OUT) :: t
     END FUNCTION

     ! generation-zone targets (the series AnalyticWaveMaker2D reads)
     INTEGER(c_int) FUNCTION ow3d_set_relax_target(handle, zone, mode, nt, dt_sample, eta, phis) &
          BIND(C, name="ow3d_set_relax_target")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       INTEGER(c_int), VALUE :: zone, mode, nt
       REAL(c_double), VALUE :: dt_sample
       REAL(c_double), DIMENSION(*), INTENT(IN) :: eta, phis
     END FUNCTION

     ! the incident wave of IncWaveType 2 on generation zone `zone` (0-based)
     INTEGER(c_int) FUNCTION ow3d_incident_wave(p, zone, nt, eta, phis, box) BIND(C, name="ow3d_incident_wave")
       IMPORT :: c_int, c_double, ow3d_params_t
       TYPE(ow3d_params_t), INTENT(IN) :: p
       INTEGER(c_int), VALUE :: zone, nt
       REAL(c_double), DIMENSION(*), INTENT(OUT) :: eta, phis
       INTEGER(c_int), DIMENSION(5), INTENT(OUT) :: box
     END FUNCTION

     ! the same wave synthesised on the device and installed as the zone's target
     INTEGER(c_int) FUNCTION ow3d_incident_wave_device(handle, zone, nt) BIND(C, name="ow3d_incident_wave_device")
       IMPORT :: c_int, c_ptr
       TYPE(c_ptr), VALUE :: handle
       INTEGER(c_int), VALUE :: zone, nt
     END FUNCTION

     ! the rollers of the breaking model after the last step (the roller.dat
     ! record of detect_breaking); pass cap = 0 to query n_rollers only
     INTEGER(c_int) FUNCTION ow3d_rollers(handle, cap, n_rollers, npts, toe, x, eta, thickness, tan_phi) &
          BIND(C, name="ow3d_rollers")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       INTEGER(c_int), VALUE :: cap
       INTEGER(c_int), INTENT(OUT) :: n_rollers
       INTEGER(c_int), DIMENSION(*), INTENT(OUT) :: npts, toe
       REAL(c_double), DIMENSION(*), INTENT(OUT) :: x, eta, thickness, tan_phi
     END FUNCTION

     ! the flux wavemaker's paddle-signal file (setupWavePaddle): call with
     ! cap = 0 for dt, nt, n2, then with y(n2) and flux(n2, nt) (time-major in C)
     INTEGER(c_int) FUNCTION ow3d_read_paddle_signal(path, cap, dt, nt, n2, y, flux) &
          BIND(C, name="ow3d_read_paddle_signal")
       IMPORT :: c_int, c_double, c_char
       CHARACTER(kind=c_char), DIMENSION(*), INTENT(IN) :: path
       INTEGER(c_int), VALUE :: cap
       REAL(c_double), INTENT(OUT) :: dt
       INTEGER(c_int), INTENT(OUT) :: nt, n2
       REAL(c_double), DIMENSION(*), INTENT(OUT) :: y, flux
     END FUNCTION

     ! install it on a handle of IncWaveType 3 (or 5) before the first step
     INTEGER(c_int) FUNCTION ow3d_set_paddle_signal(handle, nt, n2, dt, y, flux) &
          BIND(C, name="ow3d_set_paddle_signal")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       INTEGER(c_int), VALUE :: nt, n2
       REAL(c_double), VALUE :: dt
       REAL(c_double), DIMENSION(*), INTENT(IN) :: y, flux
     END FUNCTION

     ! Gauss-Seidel row order of the multigrid smoother: OW3D_SMOOTHER_LEXICOGRAPHIC
     ! gives the reference's own order (with krylov = 1, its solver's iterates)
     INTEGER(c_int) FUNCTION ow3d_set_smoother_order(handle, order) BIND(C, name="ow3d_set_smoother_order")
       IMPORT :: c_int, c_ptr
       TYPE(c_ptr), VALUE :: handle
       INTEGER(c_int), VALUE :: order
     END FUNCTION

     ! the reference's output schedule (StoreDataONOFF of the deck): EP_#####.bin
     ! or fort.NNN and OceanWave3D.end, written from the device state
     INTEGER(c_int) FUNCTION ow3d_store_data(handle, dir, nfiles) BIND(C, name="ow3d_store_data")
       IMPORT :: c_int, c_char, c_ptr
       TYPE(c_ptr), VALUE :: handle
       CHARACTER(kind=c_char), DIMENSION(*), INTENT(IN) :: dir     ! NUL-terminated, "" = cwd
       INTEGER(c_int), INTENT(OUT) :: nfiles
     END FUNCTION

     ! the deck's kinematics output (line 9, formattype 20 / 21)
     INTEGER(c_int) FUNCTION ow3d_store_kinematics(handle, dir, nfiles) BIND(C, name="ow3d_store_kinematics")
       IMPORT :: c_int, c_char, c_ptr
       TYPE(c_ptr), VALUE :: handle
       CHARACTER(kind=c_char), DIMENSION(*), INTENT(IN) :: dir
       INTEGER(c_int), INTENT(OUT) :: nfiles
     END FUNCTION

     ! u, v, w and the 9 gradient fields of the current state, whole grid
     INTEGER(c_int) FUNCTION ow3d_kinematics(handle, u, v, w, grads) BIND(C, name="ow3d_kinematics")
       IMPORT :: c_int, c_double, c_ptr
       TYPE(c_ptr), VALUE :: handle
       REAL(c_double), DIMENSION(*), INTENT(OUT) :: u, v, w, grads
     END FUNCTION

     ! message of the calling thread's last failure (NUL-terminated C string)
     TYPE(c_ptr) FUNCTION ow3d_last_error() BIND(C, name="ow3d_last_error")
       IMPORT :: c_ptr
     END FUNCTION
  END INTERFACE
END MODULE ow3d_iface
