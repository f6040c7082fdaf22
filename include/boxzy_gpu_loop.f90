! boxzy_gpu_loop.f90 -- the reference's time loop (main.f90:211-555) run by
! libboxzy_gpu.so.  A copy of main.f90 calls bx_main_loop in place of those
! lines, after init_grid, calc_eos_table, init_conditions (or read_hydro) and
! get_units, so in.nml and the ICFILES work unchanged:
!
!    call bx_main_loop(scale%rgas, step, nextstop)
!
! Between output times the steps run on the device in chunks (bx_advance_to:
! CUDA-graph runs through bx_run, the last steps before an output time one by
! one), and the state comes back only for write_files (main.f90:548-552), which
! calls state() itself on the downloaded arrays as the reference's loop would.
! Self-gravity, radiation and particles are not driven here (they stay on the
! reference's CPU path, which downloads cons, u and p every step, hands the
! force over with bx_set_gforce or bx_set_phi and uploads again).
subroutine bx_main_loop(rgas, step, nextstop)
  use iso_c_binding
  use parameters
  use grid_commons
  use boxzy_gpu
  implicit none
  real(c_double), intent(in) :: rgas        ! scale%rgas of get_units (units.f90:17)
  integer, intent(inout) :: step            ! main.f90:198-199
  real(c_double), intent(inout) :: nextstop ! main.f90:103-104
  type(bx_params) :: bp
  type(c_ptr) :: hx
  integer(c_int32_t) :: ran
  integer(c_int64_t) :: st8
  real(c_double) :: dtold8, stop_at

  bp%nx = nx; bp%ny = ny; bp%nz = nz; bp%h2stat = H2STAT
  bp%dx = dx; bp%dy = dy; bp%dz = dz; bp%cfl = cfl
  bp%small_rho = small_rho; bp%small_eps = small_eps; bp%vlimit = vlimit
  bp%gammafix = gammafix; bp%muc = muc; bp%rgas = rgas
  bp%no_outflow = merge(1, 0, [no_outflow_xl, no_outflow_xr, no_outflow_yl, &
                               no_outflow_yr, no_outflow_zl, no_outflow_zr])
  bp%fluxangmom = merge(1, 0, fluxangmom); bp%flags = 0; bp%yoffset = yoffset
  if (bx_create(bp, hx) /= 0) stop "bx_create failed"
  if (bx_upload(hx, cons, u, p) /= 0) stop "bx_upload failed"
  ! the clock of main.f90:102,196-199 (dtold starts at zero)
  if (bx_set_clock(hx, time, 0d0, int(step, c_int64_t)) /= 0) stop "bx_set_clock failed"
  do
#ifdef NOWRITEOUT
    stop_at = endtime
#else
    stop_at = nextstop
#endif
    if (bx_advance_to(hx, endtime, stop_at, ran) /= 0) then
      print *, bx_message(hx)
      stop "bx_advance_to failed"
    end if
    if (ran == 0) exit
    if (bx_get_clock(hx, time, dt, dtold8, st8) /= 0) stop "bx_get_clock failed"
    step = int(st8)
#ifndef NOWRITEOUT
    if (time >= nextstop .or. time == endtime) then
      if (bx_download(hx, cons, u, p) /= 0) stop "bx_download failed"
      call write_files(step)
      nextstop = nextstop + dtout
    end if
#endif
  end do
  ! the module arrays as the reference's loop leaves them
  if (bx_download(hx, cons, u, p) /= 0) stop "bx_download failed"
  if (bx_destroy(hx) /= 0) stop "bx_destroy failed"
end subroutine bx_main_loop
