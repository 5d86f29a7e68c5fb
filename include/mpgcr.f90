! mpgcr.f90 -- Fortran 2003 (ISO_C_BINDING) interface to the C ABI declared in mpgcr.h, for the
! reference's driver `mpsolver` (lippsLFroude_implgwopks3D_unstr3.f, cited ref.f:<line>).
!
! Compile the reference with -fdefault-real-8 -fdefault-double-8 so that REAL is C double, add
! `use mpgcr_f` to mpsolver, fill an mpg_mesh_ref with c_loc() of the COMMON arrays after
! `call input` and replace the calls on the hot path, for example
!
!     call mpdatamper(uuu, unk(1,k), k)          ->  ierr = mpg_mpdatamper(h, MPG_F_UNK+k-1, k)
!     call gcrk(prpot, unk1(1,1), unk1(1,2), unk1(1,3), uuu(1,1), uuu(1,2), uuu(1,3), imp)
!                                                ->  ierr = mpg_gcrk(h, MPG_F_PRPOT, MPG_F_UNK1,
!                                                     MPG_F_UNK1+1, MPG_F_UNK1+2, MPG_F_UUU,
!                                                     MPG_F_UUU+1, MPG_F_UUU+2, imp, st)
!
! Every function returns an integer status (MPG_OK = 0).  The derived types below are bind(C)
! copies of the C structs, member for member; tests/test_fortran_binding.py checks their member
! offsets and sizes against mpgcr.h with a C compiler (no Fortran compiler exists on the machines
! this library was built on, so the module itself is checked as text).
module mpgcr_f
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: MPG_OK = 0, MPG_ERR_ARG = 1, MPG_ERR_CUDA = 2, MPG_ERR_MESH = 3, &
       MPG_ERR_NOMEM = 4, MPG_ERR_UNSUPPORTED = 5, MPG_ERR_NUMERIC = 6
  integer(c_int), parameter :: MPG_GCR_CONVERGED = 0, MPG_GCR_STALLED = 1, MPG_GCR_MAXIT = 2, &
       MPG_GCR_NAN = 3, MPG_GCR_FALLBACK = 4
  integer(c_int), parameter :: MPG_PREC_FP64 = 0, MPG_PREC_MIXED = 1
  integer(c_int), parameter :: MPG_RESTART_TEXT = 0, MPG_RESTART_BINARY = 1
  integer(c_int), parameter :: MPG_F_UNK = 0, MPG_F_UNK1 = 16, MPG_F_UUU = 20, MPG_F_UUU0 = 23, &
       MPG_F_FRC = 26, MPG_F_UNKDASH = 30, MPG_F_PRPOT = 33, MPG_F_RHS = 34, MPG_F_COUR = 35, &
       MPG_F_ALPHA = 36, MPG_F_COEFW = 37, MPG_F_RH0 = 38, MPG_F_TH0 = 39, MPG_F_THE = 40, &
       MPG_F_DTHEDZ = 41, MPG_F_D1 = 42, MPG_F_UUU1 = 43, MPG_F_WORK = 48, MPG_F_COUNT = 56

  ! inputinc.d (ref.f:2293-2321), input_mg_v3.d (ref.f:2265-2276) and mpsolver's constants
  ! (ref.f:108-138), then this implementation's extensions
  type, bind(C) :: mpg_params
     integer(c_int) :: ntime, istst, isfera, iper
     real(c_double) :: cfl, delt
     real(c_double) :: p0inf, u0inf, v0inf, w0inf
     integer(c_int) :: ielast
     real(c_double) :: eps0
     integer(c_int) :: itr, lord
     integer(c_int) :: irl
     real(c_double) :: dxabl, dxabr, dyabd, dyabu, dzabd, dzabu
     real(c_double) :: towxl, towxr, towyd, towyu, towzd, towzu
     integer(c_int) :: mg_flag, sm_flag1
     real(c_double) :: omega
     integer(c_int) :: itrp1, itrp2
     integer(c_int) :: implgw, lipps
     real(c_double) :: strat, tetbar, g
     integer(c_int) :: iprc
     integer(c_int) :: nscal
     integer(c_int) :: precision
     integer(c_int) :: itmn
     real(c_double) :: nn_rate
     integer(c_int) :: itraj
     integer(c_int) :: itrp_c1, itrp_c2, itrp_cc
     integer(c_int) :: mg_bugs
  end type mpg_params

  ! the COMMON arrays of /n/ /xyz/ /volume/ /edg/ /wge/ /bound/ /bpoints/ /terms/ /coin/ /per2/
  ! /per4/ (ref.f:2182-2196), passed with c_loc() and their leading dimensions
  type, bind(C) :: mpg_mesh_ref
     integer(c_int) :: npoin, nedge, nbface, nboun
     integer(c_int) :: npoinx, nedgex, nfacesx
     type(c_ptr) :: coord, vol, iedge, sn, kbface, sb, ibpoin, sbb, anp
     integer(c_int) :: ncoin, ncoin2, ncoin4
     integer(c_int) :: ldcoin
     type(c_ptr) :: icoin, icoin2, icoin4
  end type mpg_mesh_ref

  ! /itero/ (ref.f:1953-1963) and the exit reason
  type, bind(C) :: mpg_gcr_stats
     integer(c_int) :: niter, nitsm, icount, status
     real(c_double) :: eer, eem
     real(c_double) :: dvmx
     real(c_double) :: rl2
     integer(c_int) :: fallbacks
     integer(c_int) :: pad
     real(c_double) :: rate
  end type mpg_gcr_stats

  ! what mpsolver prints every step (ref.f:456-459)
  type, bind(C) :: mpg_diag
     real(c_double) :: divmx, divmn, divav, divsd
     real(c_double) :: crnmx, crnmn, crnav, crnsd
     integer(c_int) :: icrnmx, niter, nitav
     integer(c_int) :: niter1
     real(c_double) :: eer, eem
     real(c_double) :: stats(16)
     real(c_double) :: mass(8)
     real(c_double) :: smin(4), smax(4)
     real(c_double) :: rate1
     integer(c_int) :: fallbacks
     integer(c_int) :: pad
  end type mpg_diag

  type, bind(C) :: mpg_info
     integer(c_int64_t) :: npoin, nedge, ncol, nedge2d
     integer(c_int) :: nlev, precision
     integer(c_int64_t) :: device_bytes
  end type mpg_info

  type, bind(C) :: mpg_ktime
     character(kind=c_char) :: name(24)
     integer(c_int64_t) :: launches
     real(c_double) :: total_ms
  end type mpg_ktime

  integer(c_int), parameter :: MPG_NOALLOC_MAX_NODES = 131072

  interface
     ! ------------------------------------------------------------ lifecycle (input, ref.f:2343-2641)
     integer(c_int) function mpg_create(prm, mesh, device, h) bind(C, name="mpg_create")
       import :: c_int, c_ptr, mpg_params, mpg_mesh_ref
       type(mpg_params), intent(in) :: prm
       type(mpg_mesh_ref), intent(in) :: mesh
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: h
     end function
     integer(c_int) function mpg_destroy(h) bind(C, name="mpg_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function mpg_analyze_mesh(mesh, info) bind(C, name="mpg_analyze_mesh")
       import :: c_int, mpg_mesh_ref, mpg_info
       type(mpg_mesh_ref), intent(in) :: mesh
       type(mpg_info), intent(out) :: info
     end function
     integer(c_int) function mpg_analyze_wide(prm, mesh, impfl, a, minv, cp) bind(C, name="mpg_analyze_wide")
       import :: c_int, c_double, mpg_params, mpg_mesh_ref
       type(mpg_params), intent(in) :: prm
       type(mpg_mesh_ref), intent(in) :: mesh
       integer(c_int), value :: impfl
       real(c_double) :: a(*), minv(*), cp(*)
     end function
     type(c_ptr) function mpg_last_error() bind(C, name="mpg_last_error")
       import :: c_ptr
     end function
     integer(c_int) function mpg_get_info(h, info) bind(C, name="mpg_get_info")
       import :: c_int, c_ptr, mpg_info
       type(c_ptr), value :: h
       type(mpg_info), intent(out) :: info
     end function
     integer(c_int) function mpg_set_coarse(h, level, mesh, match) bind(C, name="mpg_set_coarse")
       import :: c_int, c_ptr, mpg_mesh_ref
       type(c_ptr), value :: h
       integer(c_int), value :: level
       type(mpg_mesh_ref), intent(in) :: mesh
       type(c_ptr), value :: match
     end function
     integer(c_int) function mpg_set_field(h, fid, src) bind(C, name="mpg_set_field")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: fid
       real(c_double), intent(in) :: src(*)
     end function
     integer(c_int) function mpg_get_field(h, fid, dst) bind(C, name="mpg_get_field")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: fid
       real(c_double) :: dst(*)
     end function
     ! ------------------------------------------------------------ the reference's subroutines
     integer(c_int) function mpg_derivative(h, unk, out, idx) bind(C, name="mpg_derivative")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: unk, out, idx
     end function
     integer(c_int) function mpg_bcv(h, u, v, w, flag) bind(C, name="mpg_bcv")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: u, v, w
       real(c_double), value :: flag
     end function
     integer(c_int) function mpg_laplc(h, press, alap, impfl) bind(C, name="mpg_laplc")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: press, alap, impfl
     end function
     integer(c_int) function mpg_laplc_adjoint(h, y, out, impfl) bind(C, name="mpg_laplc_adjoint")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: y, out, impfl
     end function
     integer(c_int) function mpg_prfr(h, press, ustr, vstr, wstr, uout, vout, wout, impfl) bind(C, name="mpg_prfr")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: press, ustr, vstr, wstr, uout, vout, wout, impfl
     end function
     integer(c_int) function mpg_div(h, ua, va, wa, rhs, iflg, diag) bind(C, name="mpg_div")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: ua, va, wa, rhs, iflg
       type(c_ptr), value :: diag
     end function
     integer(c_int) function mpg_precon(h, rhs, p, r, iprc, impfl) bind(C, name="mpg_precon")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: rhs, p, r, iprc, impfl
     end function
     integer(c_int) function mpg_gcrk(h, p, u1, v1, w1, u2, v2, w2, impfl, stats) bind(C, name="mpg_gcrk")
       import :: c_int, c_ptr, mpg_gcr_stats
       type(c_ptr), value :: h
       integer(c_int), value :: p, u1, v1, w1, u2, v2, w2, impfl
       type(mpg_gcr_stats), intent(out) :: stats
     end function
     integer(c_int) function mpg_mpdatamper(h, unk, iflag) bind(C, name="mpg_mpdatamper")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: unk, iflag
     end function
     integer(c_int) function mpg_mpdatam(h, unk, iflag) bind(C, name="mpg_mpdatam")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: unk, iflag
     end function
     integer(c_int) function mpg_courant(h, iflag, diag) bind(C, name="mpg_courant")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: iflag
       type(c_ptr), value :: diag
     end function
     integer(c_int) function mpg_stats(h, diag) bind(C, name="mpg_stats")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, diag
     end function
     ! ------------------------------------------------------------ mpsolver (ref.f:99-463)
     integer(c_int) function mpg_setup(h, diag) bind(C, name="mpg_setup")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, diag
     end function
     integer(c_int) function mpg_step(h, diag) bind(C, name="mpg_step")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, diag
     end function
     integer(c_int) function mpg_half_forcing(h) bind(C, name="mpg_half_forcing")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function mpg_explicit_forcing(h, mtri) bind(C, name="mpg_explicit_forcing")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: mtri
     end function
     integer(c_int) function mpg_post_solve(h, mtri) bind(C, name="mpg_post_solve")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: mtri
     end function
     integer(c_int) function mpg_extrapolate(h) bind(C, name="mpg_extrapolate")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function mpg_velprd(h) bind(C, name="mpg_velprd")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function mpg_get_gcr_stats(h, stats) bind(C, name="mpg_get_gcr_stats")
       import :: c_int, c_ptr, mpg_gcr_stats
       type(c_ptr), value :: h
       type(mpg_gcr_stats), intent(out) :: stats
     end function
     integer(c_int) function mpg_synchronize(h) bind(C, name="mpg_synchronize")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
     end function
     ! ------------------------------------------------------------ learned preconditioner (iprc = 3)
     integer(c_int) function mpg_learned_init(h, seed) bind(C, name="mpg_learned_init")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: seed
     end function
     integer(c_int) function mpg_learned_set_params(h, prm, n) bind(C, name="mpg_learned_set_params")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float), intent(in) :: prm(*)
       integer(c_int), value :: n
     end function
     integer(c_int) function mpg_learned_get_params(h, prm, n) bind(C, name="mpg_learned_get_params")
       import :: c_int, c_ptr, c_float
       type(c_ptr), value :: h
       real(c_float) :: prm(*)
       integer(c_int), value :: n
     end function
     integer(c_int) function mpg_learned_forward(h, r, q) bind(C, name="mpg_learned_forward")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: r, q
     end function
     integer(c_int) function mpg_learned_loss(h, mode) bind(C, name="mpg_learned_loss")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: mode
     end function
     integer(c_int) function mpg_selftest_wait(h, arrive, spins, completed) bind(C, name="mpg_selftest_wait")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: arrive, spins
       integer(c_int), intent(out) :: completed
     end function
     integer(c_int) function mpg_learned_grad(h, r, t, grad, loss) bind(C, name="mpg_learned_grad")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: r, t
       real(c_float) :: grad(*)
       real(c_double), intent(out) :: loss
     end function
     integer(c_int) function mpg_learned_train_pair(h, r, t, lr, loss) bind(C, name="mpg_learned_train_pair")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: r, t
       real(c_float), value :: lr
       real(c_double), intent(out) :: loss
     end function
     integer(c_int) function mpg_learned_harvest(h, every, max_records) bind(C, name="mpg_learned_harvest")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: every, max_records
     end function
     integer(c_int) function mpg_learned_train_records(h, epochs, lr, mean_loss, npairs) &
          bind(C, name="mpg_learned_train_records")
       import :: c_int, c_ptr, c_float, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: epochs
       real(c_float), value :: lr
       real(c_double), intent(out) :: mean_loss
       integer(c_int), intent(out) :: npairs
     end function
     ! ------------------------------------------------------------ files (ref.f:2771-2806, 4779-4890)
     integer(c_int) function mpg_write_output(h, path, coord, npoinx) bind(C, name="mpg_write_output")
       import :: c_int, c_ptr, c_char, c_double
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
       real(c_double), intent(in) :: coord(*)
       integer(c_int), value :: npoinx
     end function
     integer(c_int) function mpg_restart_write(h, path, format, ntime) bind(C, name="mpg_restart_write")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
       integer(c_int), value :: format, ntime
     end function
     integer(c_int) function mpg_restart_read(h, path, format, ntime) bind(C, name="mpg_restart_read")
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: h
       character(kind=c_char), intent(in) :: path(*)
       integer(c_int), value :: format
       integer(c_int), intent(out) :: ntime
     end function
     ! ------------------------------------------------------------ allocation-free laplc
     integer(c_int) function mpg_laplc_noalloc(h, press, alap, impfl) bind(C, name="mpg_laplc_noalloc")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, press, alap
       integer(c_int), value :: impfl
     end function
     ! ------------------------------------------------------------ instrumentation
     integer(c_int) function mpg_get_stream(h, stream) bind(C, name="mpg_get_stream")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       type(c_ptr), intent(out) :: stream
     end function
     integer(c_int) function mpg_kernel_timing(h, enable) bind(C, name="mpg_kernel_timing")
       import :: c_int, c_ptr
       type(c_ptr), value :: h
       integer(c_int), value :: enable
     end function
     integer(c_int) function mpg_kernel_times(h, out, max, count) bind(C, name="mpg_kernel_times")
       import :: c_int, c_ptr, mpg_ktime
       type(c_ptr), value :: h
       type(mpg_ktime) :: out(*)
       integer(c_int), value :: max
       integer(c_int), intent(out) :: count
     end function
  end interface
end module mpgcr_f
