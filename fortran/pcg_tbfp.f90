! pcgMod backed by the B200 projection library (MG_MODE).
!
! A drop-in for the reference's src/pcg/pcg.f90: module pcgMod with the public
! type pcg (its public components iter_ and res_, printed by
! poissonEqn.f90:484-485) and the public procedures pcgCTOR(this, mesh, psi,
! beta) (pcg.f90:62) and solvePCG(this, mesh, psi, beta, q) (:103).  The
! settings come from the same specs/pcg_solver entries that pcgCTOR and
! multiGridCTOR read (pcg.f90:82-85, multiGrid.f90:79-86).  The solve is FP64
! PCG preconditioned by FP32 red-black Gauss-Seidel multigrid V-cycles on the
! GPU, with psi as the initial guess.  An iteration cap returns the soft status
! 1 and prints the reference's warning; errors (< 0) go to mpiABORT.
!
! Not compiled by the repository's own checks (no Fortran compiler is
! installed where the library is built).
module pcgMod
  use fieldMod
  use gridMod
  use parFileMod
  use errorHandlerMod, only: mpiABORT
  use tbfp_mod
  use, intrinsic :: iso_c_binding
  implicit none

  type, public :: pcg
    type(c_ptr), private :: h = c_null_ptr
    real(DP) :: res_
    integer :: iter_
  end type

  real(c_double), allocatable, target, private, save :: dxf_c(:), dxc_c(:), dyf_c(:), dyc_c(:), dzf_c(:), dzc_c(:)

  public :: pcgCTOR
  public :: solvePCG

contains

!========================================================================================!
  subroutine pcgCTOR(this, mesh, psi, beta)
    type(pcg) :: this
    type(grid), intent(in) :: mesh
    type(field), intent(inout) :: psi, beta
    type(parFile) :: pfile
    type(tbfp_desc) :: d
    type(tbfp_mg_params) :: prm
    integer :: n_levels, n_pre, n_post, max_iter_mg, max_iter_pcg
    real(DP) :: tol_mg, tol_pcg
    integer(c_int) :: rc

    call parFileCTOR(pfile, 'pcg_solver', 'specs')
    call readParameter(pfile, tol_pcg, 'tolPCG')
    call readParameter(pfile, max_iter_pcg, 'maxIterPCG')
    call readParameter(pfile, n_levels, 'nLevels')
    call readParameter(pfile, n_pre, 'nPreSweep')
    call readParameter(pfile, n_post, 'nPostSweep')
    call readParameter(pfile, tol_mg, 'tolMG')
    call readParameter(pfile, max_iter_mg, 'maxIterMG')

    dxf_c = mesh%dxf_(1:mesh%nx_)
    dxc_c = mesh%dxc_(1:mesh%nx_ + 1)
    dyf_c = mesh%dyf_(1:mesh%ny_)
    dyc_c = mesh%dyc_(1:mesh%ny_ + 1)
    dzf_c = mesh%dzf_(1:mesh%nz_)
    dzc_c = mesh%dzc_(1:mesh%nz_ + 1)
    d%nx = mesh%nx_
    d%ny = mesh%ny_
    d%nz = mesh%nz_
    d%hd_psi = psi%hd_
    d%hd_u = 2
    d%hd_rho = beta%hd_
    d%hd_st = 1
    d%dx_fft = mesh%xc_(2) - mesh%xc_(1)
    d%dz_fft = mesh%zc_(2) - mesh%zc_(1)
    d%dxf = c_loc(dxf_c)
    d%dxc = c_loc(dxc_c)
    d%dyf = c_loc(dyf_c)
    d%dyc = c_loc(dyc_c)
    d%dzf = c_loc(dzf_c)
    d%dzc = c_loc(dzc_c)
    d%s_Vg = s_Vg
    d%precision = TBFP_FP64
    d%tol = 1.0d-10
    d%max_iter = 8
    d%device = -1
    d%stream = c_null_ptr
    d%flags = 0
    rc = tbfp_create(d, this%h)
    if (rc < 0) call mpiABORT('pcgCTOR: tbfp_create: '//tbfp_message(rc)//' ')

    prm%n_levels = n_levels
    prm%n_pre = n_pre
    prm%n_post = n_post
    prm%tol_mg = tol_mg
    prm%max_iter_mg = max_iter_mg
    prm%tol_pcg = tol_pcg
    prm%max_iter_pcg = max_iter_pcg
    rc = tbfp_pcg_setup(this%h, prm)
    if (rc < 0) call mpiABORT('pcgCTOR: tbfp_pcg_setup: '//tbfp_message(rc)//' ')
    this%iter_ = 0
    this%res_ = 0.d0
  end subroutine
!========================================================================================!

!========================================================================================!
  ! L_beta psi = q; psi (initial guess in, solution out, ghosts updated).
  subroutine solvePCG(this, mesh, psi, beta, q)
    type(pcg), intent(inout) :: this
    type(grid), intent(in) :: mesh
    type(field), intent(inout) :: psi, beta, q
    type(tbfp_stats) :: st
    integer(c_int) :: rc

    rc = tbfp_pcg_solve(this%h, psi%f_, beta%f_, q%f_, st)
    if (rc < 0) call mpiABORT('solvePCG: tbfp_pcg_solve: '//tbfp_message(rc)//' ')
    this%iter_ = st%iterations
    this%res_ = st%rel_residual
    if (rc == TBFP_ENOTCONVERGED) write(*, '(A)') 'WARNING: max number of PCG iterations reached '  ! pcg.f90:366-373
  end subroutine
!========================================================================================!

end module pcgMod
