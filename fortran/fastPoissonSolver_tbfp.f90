! fastPoissonSolverMod backed by the B200 projection library.
!
! A drop-in for the reference's src/fastPoissonSolver/fastPoissonSolver.f90:
! the same module name, public type and public procedures with the same
! arguments -- fastPoissonSolverCTOR(this, mesh, gMesh) (fastPoissonSolver.f90:123)
! and solveFPS(this, p, s) (:337) -- so poissonEqn.f90 and main.f90 compile
! unchanged.  Build it in place of that file, with tbfp_mod.f90 compiled
! first, and add -L<repo>/tbfsolver_b200/lib -ltbfp to the link line.
!
! The library takes the whole channel on one GPU: run one MPI rank per GPU
! with px = pz = 1 (IS_PAR = .false.), or the slab form (tbfp_slab_*) for a
! channel split over ranks.  Errors (< 0) go to mpiABORT, as the reference does
! for a failed FFTW plan (fastPoissonSolver.f90:181-208).
!
! Not compiled by the repository's own checks (no Fortran compiler is
! installed where the library is built).
module fastPoissonSolverMod
  use fieldMod
  use gridMod
  use errorHandlerMod, only: mpiABORT
  use tbfp_mod
  use, intrinsic :: iso_c_binding
  implicit none

  type, public :: fastPoissonSolver
    type(c_ptr) :: h = c_null_ptr
  end type

  ! metric copies handed to tbfp_create (read at create time only)
  real(c_double), allocatable, target, private, save :: dxf_c(:), dxc_c(:), dyf_c(:), dyc_c(:), dzf_c(:), dzc_c(:)

  public :: fastPoissonSolverCTOR
  public :: solveFPS
  public :: fastPoissonSolverDTOR

contains

!========================================================================================!
  subroutine fastPoissonSolverCTOR(this, mesh, gMesh)
    type(fastPoissonSolver), intent(out) :: this
    type(grid), intent(in) :: mesh, gMesh
    type(tbfp_desc) :: d
    integer :: nxg, nyg, nzg
    integer(c_int) :: rc

    nxg = gMesh%nxg_
    nyg = gMesh%nyg_
    nzg = gMesh%nzg_
    if (mesh%nx_ /= nxg .or. mesh%ny_ /= nyg .or. mesh%nz_ /= nzg) &
      call mpiABORT('fastPoissonSolverCTOR: the GPU solver takes the whole channel on one rank ')

    dxf_c = gMesh%dxf_(1:nxg)
    dxc_c = gMesh%dxc_(1:nxg + 1)
    dyf_c = gMesh%dyf_(1:nyg)
    dyc_c = gMesh%dyc_(1:nyg + 1)
    dzf_c = gMesh%dzf_(1:nzg)
    dzc_c = gMesh%dzc_(1:nzg + 1)

    d%nx = nxg
    d%ny = nyg
    d%nz = nzg
    d%hd_psi = 1                              ! createFields_H.f90:40
    d%hd_u = 2                                ! createFields_H.f90:36
    d%hd_rho = 1                              ! createFields_H.f90:65
    d%hd_st = 1                               ! VOF.f90:175
    d%dx_fft = mesh%xc_(2) - mesh%xc_(1)      ! fastPoissonSolver.f90:222-223
    d%dz_fft = mesh%zc_(2) - mesh%zc_(1)
    d%dxf = c_loc(dxf_c)
    d%dxc = c_loc(dxc_c)
    d%dyf = c_loc(dyf_c)
    d%dyc = c_loc(dyc_c)
    d%dzf = c_loc(dzf_c)
    d%dzc = c_loc(dzc_c)
    d%s_Vg = s_Vg                             ! grid.f90:933-951
    d%precision = TBFP_FP64
    d%tol = 1.0d-10
    d%max_iter = 8
    d%device = -1                             ! the current device (one rank per GPU)
    d%stream = c_null_ptr
    d%flags = 0

    rc = tbfp_create(d, this%h)
    if (rc < 0) call mpiABORT('fastPoissonSolverCTOR: tbfp_create: '//tbfp_message(rc)//' ')
  end subroutine
!========================================================================================!

!========================================================================================!
  ! p receives the solution with its ghost cells (the updateBoundaries(p) of
  ! fastPoissonSolver.f90:381) and zero volume-weighted mean (:388-423).
  subroutine solveFPS(this, p, s)
    type(fastPoissonSolver), intent(inout) :: this
    type(field), intent(inout) :: p
    type(field), intent(in) :: s
    integer(c_int) :: rc

    rc = tbfp_solve_fps(this%h, s%f_, p%f_)
    if (rc < 0) call mpiABORT('solveFPS: tbfp_solve_fps: '//tbfp_message(rc)//' ')
  end subroutine
!========================================================================================!

!========================================================================================!
  ! No counterpart in the reference (its solver lives until the program ends):
  ! releases the device buffers.
  subroutine fastPoissonSolverDTOR(this)
    type(fastPoissonSolver), intent(inout) :: this
    integer(c_int) :: rc
    if (c_associated(this%h)) rc = tbfp_destroy(this%h)
    this%h = c_null_ptr
  end subroutine
!========================================================================================!

end module fastPoissonSolverMod
