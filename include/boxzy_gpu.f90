! boxzy_gpu.f90 -- ISO_C_BINDING interface module of libboxzy_gpu.so
! (include/boxzy_gpu.h), what a maintainer adds to the reference to drive its
! hydrodynamic step on the GPU.  The reference keeps its state in allocatable
! module arrays (grid_commons.f90:11-24); assumed-size dummies pass those
! contiguous allocatables by address, without copies.  Every interface binds
! the C prototype of the same name (checked against the header, without a
! Fortran compiler, by tests/test_host.py).
module boxzy_gpu
  use iso_c_binding
  implicit none
  type, bind(c) :: bx_params
    integer(c_int32_t) :: nx, ny, nz, h2stat
    real(c_double)     :: dx, dy, dz, cfl, small_rho, small_eps, vlimit, gammafix, muc, rgas
    integer(c_int32_t) :: no_outflow(6), fluxangmom, flags
    real(c_double)     :: yoffset
  end type
  type, bind(c) :: bx_eos_table
    integer(c_int32_t) :: neos, neos_rho
    real(c_double)     :: log_rho_eos_low, drho_eos, density_unit, tk_bgrnd
    type(c_ptr)        :: eng_table2, gamma_table2, muc_table2, tk_table2, rho_table, deng_eos_array
  end type
  interface
    ! the handle (init_grid and the module arrays; cleanup)
    integer(c_int) function bx_create(p, h) bind(c, name="bx_create")
      import; type(bx_params), intent(in) :: p; type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function bx_destroy(h) bind(c, name="bx_destroy")
      import; type(c_ptr), value :: h
    end function
    type(c_ptr) function bx_last_error(h) bind(c, name="bx_last_error")
      import; type(c_ptr), value :: h
    end function
    ! the module arrays in and out, the clock
    integer(c_int) function bx_upload(h, cons, u, p) bind(c, name="bx_upload")
      import; type(c_ptr), value :: h; real(c_double), intent(in) :: cons(*), u(*), p(*)
    end function
    integer(c_int) function bx_upload_conserved(h, cons) bind(c, name="bx_upload_conserved")
      import; type(c_ptr), value :: h; real(c_double), intent(in) :: cons(*)
    end function
    integer(c_int) function bx_download(h, cons, u, p) bind(c, name="bx_download")
      import; type(c_ptr), value :: h; real(c_double), intent(out) :: cons(*), u(*), p(*)
    end function
    integer(c_int) function bx_set_clock(h, t, dtold, step) bind(c, name="bx_set_clock")
      import; type(c_ptr), value :: h; real(c_double), value :: t, dtold
      integer(c_int64_t), value :: step
    end function
    integer(c_int) function bx_get_clock(h, t, dt, dtold, step) bind(c, name="bx_get_clock")
      import; type(c_ptr), value :: h; real(c_double), intent(out) :: t, dt, dtold
      integer(c_int64_t), intent(out) :: step
    end function
    ! the loop body
    integer(c_int) function bx_step(h, endtime, ran) bind(c, name="bx_step")
      import; type(c_ptr), value :: h; real(c_double), value :: endtime
      integer(c_int32_t), intent(out) :: ran
    end function
    integer(c_int) function bx_step_host(h, cons_in, cons_out, endtime, ran) &
        bind(c, name="bx_step_host")
      import; type(c_ptr), value :: h; real(c_double), intent(in) :: cons_in(*)
      real(c_double), intent(inout) :: cons_out(*); real(c_double), value :: endtime
      integer(c_int32_t), intent(out) :: ran
    end function
    integer(c_int) function bx_run(h, endtime, nsteps, steps_taken) bind(c, name="bx_run")
      import; type(c_ptr), value :: h; real(c_double), value :: endtime
      integer(c_int64_t), value :: nsteps; integer(c_int64_t), intent(out) :: steps_taken
    end function
    integer(c_int) function bx_status(h, bits, last_path) bind(c, name="bx_status")
      import; type(c_ptr), value :: h; integer(c_int32_t), intent(out) :: bits, last_path
    end function
    ! forces and the tabulated EOS
    integer(c_int) function bx_set_gforce(h, g) bind(c, name="bx_set_gforce")
      import; type(c_ptr), value :: h; real(c_double), intent(in) :: g(*)
    end function
    integer(c_int) function bx_set_phi(h, phi) bind(c, name="bx_set_phi")
      import; type(c_ptr), value :: h; real(c_double), intent(in) :: phi(*)
    end function
    ! the same two with an address, so c_null_ptr removes the force
    integer(c_int) function bx_set_gforce_ptr(h, g) bind(c, name="bx_set_gforce")
      import; type(c_ptr), value :: h, g
    end function
    integer(c_int) function bx_set_phi_ptr(h, phi) bind(c, name="bx_set_phi")
      import; type(c_ptr), value :: h, phi
    end function
    integer(c_int) function bx_set_eos_table(h, t) bind(c, name="bx_set_eos_table")
      import; type(c_ptr), value :: h; type(bx_eos_table), intent(in) :: t
    end function
    ! celldump files (write_files, read_hydro); path ends with c_null_char
    integer(c_int) function bx_write_celldump(h, path, phi) bind(c, name="bx_write_celldump")
      import; type(c_ptr), value :: h; character(kind=c_char), intent(in) :: path(*)
      real(c_double), intent(in) :: phi(*)
    end function
    integer(c_int) function bx_read_celldump(h, path, phi, t, step) &
        bind(c, name="bx_read_celldump")
      import; type(c_ptr), value :: h; character(kind=c_char), intent(in) :: path(*)
      real(c_double), intent(out) :: phi(*), t; integer(c_int64_t), intent(out) :: step
    end function
    ! the loop's subroutines one by one, for bisection against the reference
    integer(c_int) function bx_state(h) bind(c, name="bx_state")
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function bx_velocity(h) bind(c, name="bx_velocity")
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function bx_courant(h, dt) bind(c, name="bx_courant")
      import; type(c_ptr), value :: h; real(c_double), intent(out) :: dt
    end function
    integer(c_int) function bx_source(h, siter) bind(c, name="bx_source")
      import; type(c_ptr), value :: h; integer(c_int32_t), value :: siter
    end function
    integer(c_int) function bx_ghost(h) bind(c, name="bx_ghost")
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function bx_flux(h, avg) bind(c, name="bx_flux")
      import; type(c_ptr), value :: h; integer(c_int32_t), value :: avg
    end function
    integer(c_int) function bx_avisc(h) bind(c, name="bx_avisc")
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function bx_set_avmag(h, ax, ay, az) bind(c, name="bx_set_avmag")
      import; type(c_ptr), value :: h; real(c_double), value :: ax, ay, az
    end function
    integer(c_int) function bx_download_qq(h, qq) bind(c, name="bx_download_qq")
      import; type(c_ptr), value :: h; real(c_double), intent(out) :: qq(*)
    end function
    integer(c_int) function bx_save_cons_old(h) bind(c, name="bx_save_cons_old")
      import; type(c_ptr), value :: h
    end function
    integer(c_int) function bx_set_dt(h, dt) bind(c, name="bx_set_dt")
      import; type(c_ptr), value :: h; real(c_double), value :: dt
    end function
  end interface
contains
  ! the message of the last failed call on h, as a Fortran string
  function bx_message(h) result(msg)
    type(c_ptr), intent(in) :: h
    character(len=:), allocatable :: msg
    character(kind=c_char), pointer :: c(:)
    integer :: i, n
    call c_f_pointer(bx_last_error(h), c, [4096])
    n = 0
    do while (c(n + 1) /= c_null_char)
      n = n + 1
    end do
    allocate(character(len=n) :: msg)
    do i = 1, n
      msg(i:i) = c(i)
    end do
  end function

  ! Advances the run to the end of the first step whose time reaches stoptime
  ! (the step after which the reference's loop writes its output,
  ! main.f90:549-552), or to endtime.  dt grows by at most a factor 1.1 per step
  ! (main.f90:270), so while even that growth from the last step's dt cannot
  ! reach stoptime, the steps go in chunks through bx_run (CUDA graphs, no host
  ! round trip per step); the last steps before stoptime go one by one through
  ! bx_step, so the run stops exactly where the reference's loop writes.  The
  ! bound is evaluated with the device's own operations (dt*1.1, time+dt),
  ! which round monotonically, so no chunk can cross stoptime.  ran = 0 when
  ! the loop had already ended (time >= endtime or the step cap of main.f90:212).
  integer(c_int) function bx_advance_to(h, endtime, stoptime, ran) result(rc)
    type(c_ptr), intent(in) :: h
    real(c_double), intent(in) :: endtime, stoptime
    integer(c_int32_t), intent(out) :: ran
    real(c_double) :: t, dt, dtold, tt, d
    integer(c_int64_t) :: st, k, taken
    integer(c_int32_t) :: r1
    ran = 0
    do
      rc = bx_get_clock(h, t, dt, dtold, st)
      if (rc /= 0) return
      k = 0
      if (st > 0 .and. dtold > 0d0) then
        tt = t
        d = dtold
        do while (k < 256)
          d = d * 1.1d0
          if (tt + d >= stoptime) exit
          tt = tt + d
          k = k + 1
        end do
      end if
      if (k > 0) then
        rc = bx_run(h, endtime, k, taken)
        if (rc /= 0) return
        if (taken > 0) ran = 1
        if (taken < k) return
      else
        rc = bx_step(h, endtime, r1)
        if (rc /= 0) return
        if (r1 == 0) return
        ran = 1
        rc = bx_get_clock(h, t, dt, dtold, st)
        if (rc /= 0) return
        if (t >= stoptime .or. t == endtime) return
      end if
    end do
  end function
end module boxzy_gpu
