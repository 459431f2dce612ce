! bgk_c.f90 -- ISO_C_BINDING interface to libbgkpcm (include/bgk_pcm.h) for a
! Fortran host such as the reference's STEP_7/main.f90.  The reference's own
! C interop (STEP_7/get_mem_mod.f90:7 binding STEP_7/get_mem.c:23) uses the
! same style.  Arrays are passed in the reference layout (0:Nx+1, 0:Ny+1),
! leading dimension Nx+2.
module bgk_c
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: BGK_OK = 0
  integer(c_int), parameter :: BGK_ERR_ARG = -1, BGK_ERR_UNSUPPORTED = -2, BGK_ERR_CUDA = -3, &
                               BGK_ERR_OOM = -4, BGK_ERR_STATE = -5, BGK_ERR_IO = -6, BGK_ERR_NONFINITE = -7
  integer(c_int), parameter :: BGK_PREC_F64 = 0, BGK_PREC_F32 = 1, BGK_PREC_F16 = 2, BGK_PREC_F32X = 3
  integer(c_int), parameter :: BGK_TANH_PORTABLE = 0, BGK_TANH_DEVICE = 1
  integer(c_int), parameter :: BGK_HEAT_WEST = 0, BGK_HEAT_RIGHT = 1, BGK_HEAT_BOTTOM = 2
  integer(c_int), parameter :: BGK_FIELD_F0 = 0, BGK_FIELD_G0 = 9
  integer(c_int), parameter :: BGK_FIELD_RHO = 18, BGK_FIELD_T = 19, BGK_FIELD_U = 20, BGK_FIELD_V = 21
  integer(c_int), parameter :: BGK_FIELD_PHI = 22, BGK_FIELD_PHI_PREC = 23
  integer(c_int), parameter :: BGK_FIELD_RHO2 = 24, BGK_FIELD_T2 = 25, BGK_FIELD_U2 = 26, BGK_FIELD_V2 = 27
  integer(c_int), parameter :: BGK_FIELD_FP0 = 28, BGK_FIELD_GP0 = 37, BGK_NFIELDS = 46
  integer(c_int), parameter :: BGK_STATIC_SUMS_MAX_NY = 32768

  type, bind(c) :: bgk_params
     integer(c_int) :: iter, noutput, dump, Nx, Ny
     real(c_double) :: Re, rho0, rho1, tau_f, tau_g, T0, T_in_sol, grav, eps, &
                       stefan_number, T_width, length
     integer(c_int) :: westBC, eastBC, northBC, southBC
  end type bgk_params

  type, bind(c) :: bgk_adjoint_spec
     integer(c_int) :: nsteps, checkpoint_every, nprobes
     type(c_ptr) :: probe_i, probe_j, phi_target
  end type bgk_adjoint_spec

  type, bind(c) :: bgk_options
     integer(c_int) :: precision, tanh_mode, fma, device, smooth, heat
  end type bgk_options

  interface
     function bgk_read_input(path, p) bind(c, name="bgk_read_input") result(rc)
       import :: c_int, c_char, bgk_params
       character(kind=c_char), dimension(*), intent(in) :: path
       type(bgk_params), intent(out) :: p
       integer(c_int) :: rc
     end function
     function bgk_create(p, opt, ctx) bind(c, name="bgk_create") result(rc)
       import :: c_int, c_ptr, bgk_params, bgk_options
       type(bgk_params), intent(in) :: p
       type(bgk_options), intent(in) :: opt
       type(c_ptr), intent(out) :: ctx
       integer(c_int) :: rc
     end function
     function bgk_destroy(ctx) bind(c, name="bgk_destroy") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_initialize(ctx) bind(c, name="bgk_initialize") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_step(ctx, nsteps) bind(c, name="bgk_step") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: nsteps
       integer(c_int) :: rc
     end function
     ! one per reference subroutine (STEP_7/main.f90:60-69)
     function bgk_bc_f(ctx) bind(c, name="bgk_bc_f") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_bc_g(ctx) bind(c, name="bgk_bc_g") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_streaming(ctx) bind(c, name="bgk_streaming") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_moments_pre(ctx) bind(c, name="bgk_moments_pre") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_phase_field(ctx) bind(c, name="bgk_phase_field") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_forces(ctx) bind(c, name="bgk_forces") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_collision(ctx) bind(c, name="bgk_collision") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_moments(ctx) bind(c, name="bgk_moments") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_upload(ctx, field, host, ld) bind(c, name="bgk_upload") result(rc)
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: field, ld
       real(c_double), dimension(*), intent(in) :: host
       integer(c_int) :: rc
     end function
     function bgk_download(ctx, field, host, ld) bind(c, name="bgk_download") result(rc)
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: field, ld
       real(c_double), dimension(*), intent(out) :: host
       integer(c_int) :: rc
     end function
     function bgk_download_region(ctx, field, i0, j0, ni, nj, host, ld) bind(c, name="bgk_download_region") result(rc)
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: field, i0, j0, ni, nj, ld
       real(c_double), dimension(*), intent(out) :: host
       integer(c_int) :: rc
     end function
     function bgk_field_sums(ctx, out) bind(c, name="bgk_field_sums") result(rc)
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), dimension(4), intent(out) :: out
       integer(c_int) :: rc
     end function
     function bgk_get_it(ctx, it) bind(c, name="bgk_get_it") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), intent(out) :: it
       integer(c_int) :: rc
     end function
     function bgk_set_it(ctx, it) bind(c, name="bgk_set_it") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: it
       integer(c_int) :: rc
     end function
     function bgk_set_tin(ctx, tin, ny) bind(c, name="bgk_set_tin") result(rc)
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), dimension(*), intent(in) :: tin
       integer(c_int), value :: ny
       integer(c_int) :: rc
     end function
     function bgk_sync(ctx) bind(c, name="bgk_sync") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int) :: rc
     end function
     function bgk_save(ctx, path) bind(c, name="bgk_save") result(rc)
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char), dimension(*), intent(in) :: path
       integer(c_int) :: rc
     end function
     function bgk_load(ctx, path) bind(c, name="bgk_load") result(rc)
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char), dimension(*), intent(in) :: path
       integer(c_int) :: rc
     end function
     function bgk_adjoint_run(ctx, spec, loss, grad_tin, grad_tau_g) bind(c, name="bgk_adjoint_run") result(rc)
       import :: c_int, c_ptr, c_double, bgk_adjoint_spec
       type(c_ptr), value :: ctx
       type(bgk_adjoint_spec), intent(in) :: spec
       real(c_double), intent(out) :: loss, grad_tau_g
       real(c_double), dimension(*), intent(out) :: grad_tin
       integer(c_int) :: rc
     end function
     function bgk_get_stream(ctx, stream) bind(c, name="bgk_get_stream") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       type(c_ptr), intent(out) :: stream
       integer(c_int) :: rc
     end function
     ! y-slab decomposition: steps between halo exchanges and the packed
     ! ghost rows (device buffers, e.g. from the host's MPI/NCCL layer)
     function bgk_advance(ctx, nsteps) bind(c, name="bgk_advance") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: nsteps
       integer(c_int) :: rc
     end function
     function bgk_rows_bytes(ctx, nrows, bytes) bind(c, name="bgk_rows_bytes") result(rc)
       import :: c_int, c_ptr, c_size_t
       type(c_ptr), value :: ctx
       integer(c_int), value :: nrows
       integer(c_size_t), intent(out) :: bytes
       integer(c_int) :: rc
     end function
     function bgk_rows_pack(ctx, j0, nrows, dev_buf) bind(c, name="bgk_rows_pack") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, dev_buf
       integer(c_int), value :: j0, nrows
       integer(c_int) :: rc
     end function
     function bgk_rows_unpack(ctx, j0, nrows, dev_buf) bind(c, name="bgk_rows_unpack") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, dev_buf
       integer(c_int), value :: j0, nrows
       integer(c_int) :: rc
     end function
     function bgk_field_sums_rows(ctx, j0, nrows, sums) bind(c, name="bgk_field_sums_rows") result(rc)
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: j0, nrows
       real(c_double), dimension(4), intent(out) :: sums
       integer(c_int) :: rc
     end function
     ! interior sums over the caller's own device arrays, with no allocation
     ! (rho, T, phi, out: device addresses, e.g. from CUDA Fortran's c_devloc)
     function bgk_field_sums_static(rho, T, phi, Nx, Ny, ld, stream, out) &
          bind(c, name="bgk_field_sums_static") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: rho, T, phi
       integer(c_int), value :: Nx, Ny, ld
       type(c_ptr), value :: stream, out
       integer(c_int) :: rc
     end function
     function bgk_last_error() bind(c, name="bgk_last_error") result(msg)
       import :: c_ptr
       type(c_ptr) :: msg
     end function
  end interface
end module bgk_c
