! tbfp_mod -- ISO_C_BINDING interface to the B200 projection library (include/tbfp.h).
!
! Every type and entry point of tbfp.h, declared for Fortran 2003 callers.
! Arrays are passed as the caller's allocatables with their halos (assumed
! size, f(1-hd:nx+hd, ...) column-major), exactly as the reference allocates
! them (field.f90:271-273).  Optional array-of-pointer arguments (the surface-
! tension components st_n, st_nm1, st) are type(c_ptr), value: pass c_null_ptr
! for none, or c_loc of a type(c_ptr) :: p(3) holding c_loc of each component.
!
! This file is not compiled in the repository's own checks (no Fortran
! compiler is installed where the library is built); the C declarations it
! mirrors are compiled by tests/c/tbfp_abi_check.c.  Link with
! -L<repo>/tbfsolver_b200/lib -ltbfp next to -lfftw3 in the reference's Makefile.
module tbfp_mod
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: TBFP_OK = 0, TBFP_ENOTCONVERGED = 1
  integer(c_int), parameter :: TBFP_EINVAL = -1, TBFP_ENULL = -2, TBFP_ECUDA = -3, TBFP_ENOMEM = -4
  integer(c_int), parameter :: TBFP_EUNSUPPORTED = -5, TBFP_ENODEVICE = -6, TBFP_ENONFINITE = -7
  integer(c_int), parameter :: TBFP_ESINGULAR = -8
  integer(c_int), parameter :: TBFP_FP64 = 0, TBFP_MIXED = 1
  integer(c_int), parameter :: TBFP_FLAG_ASYNC = 1, TBFP_FLAG_TIMING = 2, TBFP_FLAG_RESIDUAL = 4

  type, bind(C) :: tbfp_desc
    integer(c_int) :: nx, ny, nz
    integer(c_int) :: hd_psi, hd_u, hd_rho, hd_st
    real(c_double) :: dx_fft, dz_fft
    type(c_ptr)    :: dxf, dxc, dyf, dyc, dzf, dzc
    real(c_double) :: s_Vg
    integer(c_int) :: precision
    real(c_double) :: tol
    integer(c_int) :: max_iter
    integer(c_int) :: device
    type(c_ptr)    :: stream
    integer(c_int) :: flags            ! unsigned int in C; the flags are small
  end type

  type, bind(C) :: tbfp_stats
    integer(c_int) :: iterations
    real(c_double) :: rel_residual, max_div, cont_err, ms_device
    real(c_double) :: ms_stage(8)
  end type

  type, bind(C) :: tbfp_mg_params
    integer(c_int) :: n_levels, n_pre, n_post
    real(c_double) :: tol_mg
    integer(c_int) :: max_iter_mg
    real(c_double) :: tol_pcg
    integer(c_int) :: max_iter_pcg
  end type

  type, bind(C) :: tbfp_vof_desc
    type(c_ptr)    :: xc, yc, zc, xf, yf, zf
    real(c_double) :: rhol, rhog, mul, mug
  end type

  type, bind(C) :: tbfp_momentum_desc
    integer(c_int) :: scheme
    real(c_double) :: gch, g
    type(c_ptr)    :: dxf, dxc, dyf, dyc, dzf, dzc, yc, yf
    real(c_double) :: ubot(3), utop(3)
  end type

  type, bind(C) :: tbfp_member_io
    type(c_ptr) :: ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi_n, psi_nm1, psi
  end type

  interface
    ! --- lifecycle ----------------------------------------------------------
    integer(c_int) function tbfp_abi_version() bind(C, name='tbfp_abi_version')
      import
    end function
    type(c_ptr) function tbfp_strerror(status) bind(C, name='tbfp_strerror')
      import; integer(c_int), value :: status
    end function
    type(c_ptr) function tbfp_last_error(h) bind(C, name='tbfp_last_error')
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function tbfp_create(d, h) bind(C, name='tbfp_create')
      import; type(tbfp_desc), intent(in) :: d; type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function tbfp_destroy(h) bind(C, name='tbfp_destroy')
      import; type(c_ptr), value :: h
    end function
    integer(c_size_t) function tbfp_device_bytes(h) bind(C, name='tbfp_device_bytes')
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function tbfp_get_stats(h, stats) bind(C, name='tbfp_get_stats')
      import; type(c_ptr), value :: h; type(tbfp_stats), intent(out) :: stats
    end function
    integer(c_int) function tbfp_set_wait_limit(h, cycles) bind(C, name='tbfp_set_wait_limit')
      import; type(c_ptr), value :: h; integer(c_long_long), value :: cycles
    end function

    ! --- solveFPS, computeSource, makeVelocityDivFree, continuity error --------
    integer(c_int) function tbfp_solve_fps(h, s, psi) bind(C, name='tbfp_solve_fps')
      import; type(c_ptr), value :: h; real(c_double) :: s(*), psi(*)
    end function
    integer(c_int) function tbfp_solve_fps_dev(h, s, psi) bind(C, name='tbfp_solve_fps_dev')
      import; type(c_ptr), value :: h, s, psi
    end function
    integer(c_int) function tbfp_rhs_split(h, ux, uy, uz, rho, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0, s) &
        bind(C, name='tbfp_rhs_split')
      import; type(c_ptr), value :: h
      real(c_double) :: ux(*), uy(*), uz(*), rho(*), psi_n(*), psi_nm1(*), s(*)
      type(c_ptr), value :: st_n, st_nm1
      real(c_double), value :: dt, alpha, rho0
    end function
    integer(c_int) function tbfp_rhs_split_dev(h, ux, uy, uz, rho, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0, s) &
        bind(C, name='tbfp_rhs_split_dev')
      import; type(c_ptr), value :: h, ux, uy, uz, rho, psi_n, psi_nm1, st_n, st_nm1, s
      real(c_double), value :: dt, alpha, rho0
    end function
    integer(c_int) function tbfp_correct(h, ux, uy, uz, psi, psi_n, psi_nm1, rho, st_n, st_nm1, dt, alpha, rho0) &
        bind(C, name='tbfp_correct')
      import; type(c_ptr), value :: h
      real(c_double) :: ux(*), uy(*), uz(*), psi(*), psi_n(*), psi_nm1(*), rho(*)
      type(c_ptr), value :: st_n, st_nm1
      real(c_double), value :: dt, alpha, rho0
    end function
    integer(c_int) function tbfp_correct_dev(h, ux, uy, uz, psi, psi_n, psi_nm1, rho, st_n, st_nm1, dt, alpha, &
                                             rho0) bind(C, name='tbfp_correct_dev')
      import; type(c_ptr), value :: h, ux, uy, uz, psi, psi_n, psi_nm1, rho, st_n, st_nm1
      real(c_double), value :: dt, alpha, rho0
    end function
    integer(c_int) function tbfp_continuity_error(h, ux, uy, uz, dt, max_div, cont_err) &
        bind(C, name='tbfp_continuity_error')
      import; type(c_ptr), value :: h
      real(c_double) :: ux(*), uy(*), uz(*)
      real(c_double), value :: dt
      real(c_double), intent(out) :: max_div, cont_err
    end function
    integer(c_int) function tbfp_continuity_error_dev(h, ux, uy, uz, dt, max_div, cont_err) &
        bind(C, name='tbfp_continuity_error_dev')
      import; type(c_ptr), value :: h, ux, uy, uz
      real(c_double), value :: dt
      real(c_double), intent(out) :: max_div, cont_err
    end function
    integer(c_int) function tbfp_projection(h, ux, uy, uz, rho, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0, &
                                            psi, stats) bind(C, name='tbfp_projection')
      import; type(c_ptr), value :: h
      real(c_double) :: ux(*), uy(*), uz(*), rho(*), psi_n(*), psi_nm1(*), psi(*)
      type(c_ptr), value :: st_n, st_nm1
      real(c_double), value :: dt, alpha, rho0
      type(tbfp_stats) :: stats
    end function
    integer(c_int) function tbfp_projection_dev(h, ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi_n, &
                                                psi_nm1, st_n, st_nm1, dt, alpha, rho0, psi, stats) &
        bind(C, name='tbfp_projection_dev')
      import; type(c_ptr), value :: h, ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi_n, psi_nm1
      type(c_ptr), value :: st_n, st_nm1, psi
      real(c_double), value :: dt, alpha, rho0
      type(tbfp_stats) :: stats
    end function

    ! --- MG_MODE ------------------------------------------------------------
    integer(c_int) function tbfp_pcg_setup(h, p) bind(C, name='tbfp_pcg_setup')
      import; type(c_ptr), value :: h; type(tbfp_mg_params), intent(in) :: p
    end function
    integer(c_int) function tbfp_pcg_solve(h, psi, beta, q, stats) bind(C, name='tbfp_pcg_solve')
      import; type(c_ptr), value :: h
      real(c_double) :: psi(*), beta(*), q(*)
      type(tbfp_stats) :: stats
    end function
    integer(c_int) function tbfp_pcg_solve_dev(h, psi, beta, q, stats) bind(C, name='tbfp_pcg_solve_dev')
      import; type(c_ptr), value :: h, psi, beta, q
      type(tbfp_stats) :: stats
    end function
    integer(c_int) function tbfp_projection_mg(h, ux, uy, uz, rho, dt, alpha, psi, stats) &
        bind(C, name='tbfp_projection_mg')
      import; type(c_ptr), value :: h
      real(c_double) :: ux(*), uy(*), uz(*), rho(*), psi(*)
      real(c_double), value :: dt, alpha
      type(tbfp_stats) :: stats
    end function
    integer(c_int) function tbfp_projection_mg_dev(h, ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, dt, &
                                                   alpha, psi, stats) bind(C, name='tbfp_projection_mg_dev')
      import; type(c_ptr), value :: h, ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi
      real(c_double), value :: dt, alpha
      type(tbfp_stats) :: stats
    end function

    ! --- material properties, momentum predictor, boundaries, flow control ----
    integer(c_int) function tbfp_vof_setup(h, v) bind(C, name='tbfp_vof_setup')
      import; type(c_ptr), value :: h; type(tbfp_vof_desc), intent(in) :: v
    end function
    integer(c_int) function tbfp_material_props(h, c, cs, rho, mu) bind(C, name='tbfp_material_props')
      import; type(c_ptr), value :: h; real(c_double) :: c(*), cs(*), rho(*), mu(*)
    end function
    integer(c_int) function tbfp_material_props_dev(h, c, cs, rho, mu) bind(C, name='tbfp_material_props_dev')
      import; type(c_ptr), value :: h, c, cs, rho, mu
    end function
    integer(c_int) function tbfp_material_props_pass_dev(h, inp, out, rho, mu) &
        bind(C, name='tbfp_material_props_pass_dev')
      import; type(c_ptr), value :: h, inp, out, rho, mu
    end function
    integer(c_int) function tbfp_momentum_setup(h, m) bind(C, name='tbfp_momentum_setup')
      import; type(c_ptr), value :: h; type(tbfp_momentum_desc), intent(in) :: m
    end function
    integer(c_int) function tbfp_momentum_fluxes(h, phi_x, phi_y, phi_z, set) bind(C, name='tbfp_momentum_fluxes')
      import; type(c_ptr), value :: h; real(c_double) :: phi_x(*), phi_y(*), phi_z(*)
      integer(c_int), value :: set
    end function
    integer(c_int) function tbfp_momentum_predictor(h, ux, uy, uz, c, mu, rho, st, dt, alpha, gamma, xi, rho0, fs) &
        bind(C, name='tbfp_momentum_predictor')
      import; type(c_ptr), value :: h
      real(c_double) :: ux(*), uy(*), uz(*), c(*), mu(*), rho(*)
      type(c_ptr), value :: st
      real(c_double), value :: dt, alpha, gamma, xi, rho0, fs
    end function
    integer(c_int) function tbfp_momentum_predictor_dev(h, ux, uy, uz, c, mu, rho, st, dt, alpha, gamma, xi, rho0, &
                                                        fs) bind(C, name='tbfp_momentum_predictor_dev')
      import; type(c_ptr), value :: h, ux, uy, uz, c, mu, rho, st
      real(c_double), value :: dt, alpha, gamma, xi, rho0, fs
    end function
    integer(c_int) function tbfp_momentum_predictor_out_dev(h, ux, uy, uz, ux_out, uy_out, uz_out, c, mu, rho, st, &
                                                            dt, alpha, gamma, xi, rho0, fs) &
        bind(C, name='tbfp_momentum_predictor_out_dev')
      import; type(c_ptr), value :: h, ux, uy, uz, ux_out, uy_out, uz_out, c, mu, rho, st
      real(c_double), value :: dt, alpha, gamma, xi, rho0, fs
    end function
    integer(c_int) function tbfp_update_boundaries_v(h, ux, uy, uz) bind(C, name='tbfp_update_boundaries_v')
      import; type(c_ptr), value :: h; real(c_double) :: ux(*), uy(*), uz(*)
    end function
    integer(c_int) function tbfp_update_boundaries_v_dev(h, ux, uy, uz) bind(C, name='tbfp_update_boundaries_v_dev')
      import; type(c_ptr), value :: h, ux, uy, uz
    end function
    integer(c_int) function tbfp_rho_face_sum(h, rho, s) bind(C, name='tbfp_rho_face_sum')
      import; type(c_ptr), value :: h; real(c_double) :: rho(*); real(c_double), intent(out) :: s
    end function
    integer(c_int) function tbfp_rho_face_sum_dev(h, rho, s) bind(C, name='tbfp_rho_face_sum_dev')
      import; type(c_ptr), value :: h, rho; real(c_double), intent(out) :: s
    end function
    integer(c_int) function tbfp_flow_rate(h, ux, q) bind(C, name='tbfp_flow_rate')
      import; type(c_ptr), value :: h; real(c_double) :: ux(*); real(c_double), intent(out) :: q
    end function
    integer(c_int) function tbfp_flow_rate_dev(h, ux, q) bind(C, name='tbfp_flow_rate_dev')
      import; type(c_ptr), value :: h, ux; real(c_double), intent(out) :: q
    end function
    integer(c_int) function tbfp_add_ux(h, ux, uf) bind(C, name='tbfp_add_ux')
      import; type(c_ptr), value :: h; real(c_double) :: ux(*); real(c_double), value :: uf
    end function
    integer(c_int) function tbfp_add_ux_dev(h, ux, uf) bind(C, name='tbfp_add_ux_dev')
      import; type(c_ptr), value :: h, ux; real(c_double), value :: uf
    end function

    ! --- slab form, ensemble, allocation-free solve ----------------------------
    integer(c_int) function tbfp_slab_create(d, nz_total, k0, kx0, nkx_loc, h) bind(C, name='tbfp_slab_create')
      import; type(tbfp_desc), intent(in) :: d; integer(c_int), value :: nz_total, k0, kx0, nkx_loc
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function tbfp_slab_forward_x(h, s, spec_z) bind(C, name='tbfp_slab_forward_x')
      import; type(c_ptr), value :: h, s, spec_z
    end function
    integer(c_int) function tbfp_slab_spectral(h, spec_x) bind(C, name='tbfp_slab_spectral')
      import; type(c_ptr), value :: h, spec_x
    end function
    integer(c_int) function tbfp_slab_inverse_x(h, spec_z, psi) bind(C, name='tbfp_slab_inverse_x')
      import; type(c_ptr), value :: h, spec_z, psi
    end function
    integer(c_int) function tbfp_ensemble_create(n, descs, nstreams, e) bind(C, name='tbfp_ensemble_create')
      import; integer(c_int), value :: n, nstreams; type(tbfp_desc), intent(in) :: descs(*)
      type(c_ptr), intent(out) :: e
    end function
    integer(c_int) function tbfp_ensemble_destroy(e) bind(C, name='tbfp_ensemble_destroy')
      import; type(c_ptr), value :: e
    end function
    integer(c_int) function tbfp_ensemble_size(e) bind(C, name='tbfp_ensemble_size')
      import; type(c_ptr), value :: e
    end function
    integer(c_int) function tbfp_ensemble_projection_dev(e, io, dt, alpha, rho0, stats) &
        bind(C, name='tbfp_ensemble_projection_dev')
      import; type(c_ptr), value :: e; type(tbfp_member_io), intent(in) :: io(*)
      real(c_double), value :: dt, alpha, rho0
      type(tbfp_stats) :: stats(*)
    end function
    integer(c_int) function tbfp_solve_fps_noalloc(d, s, psi) bind(C, name='tbfp_solve_fps_noalloc')
      import; type(tbfp_desc), intent(in) :: d; type(c_ptr), value :: s, psi
    end function
  end interface

contains

  ! The message of a status code as a Fortran string (for mpiABORT).
  function tbfp_message(status) result(msg)
    integer(c_int), intent(in) :: status
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    character(kind=c_char), pointer :: c(:)
    integer :: n
    p = tbfp_strerror(status)
    call c_f_pointer(p, c, [256])
    n = 0
    do while (n < 256)
      if (c(n + 1) == c_null_char) exit
      n = n + 1
    end do
    allocate(character(len=n) :: msg)
    msg = transfer(c(1:n), msg)
  end function

end module tbfp_mod
