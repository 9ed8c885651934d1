! fwt_iface.f90 -- iso_c_binding interface of libfwt (include/fwt.h) for a Fortran host that
! keeps the reference program's input reading and replaces its construction and statistics
! loops (tube.f90:392-1188) with calls into the CUDA library.  Not built here (no Fortran
! compiler in this image); the C++ driver fastweavturb_b200/driver/fwt_tube_main.cpp is the
! shipped host.
module fwt_iface
   use iso_c_binding
   implicit none

   type, bind(C) :: fwt_params
      integer(c_int)    :: N, N_downsample, line_s, line_e
      real(c_double)    :: sigma_ratio, eta_t
      integer(c_int)    :: ntf_times, ntf_pre
      real(c_double)    :: Rtube_ratio, dzeta_sup
      integer(c_int)    :: precision, deposit_mode, device
      type(c_ptr)       :: stream
      integer(c_int)    :: if_pdf, if_Sp, Sp_order, pdf_bins, vorticity_output
      integer(c_size_t) :: mem_cap
   end type fwt_params

   interface
      integer(c_int) function fwt_default_params(p) bind(C, name="fwt_default_params")
         import :: c_int, fwt_params
         type(fwt_params) :: p
      end function
      integer(c_int) function fwt_create(p, ctx) bind(C, name="fwt_create")
         import :: c_int, c_ptr, fwt_params
         type(fwt_params) :: p
         type(c_ptr) :: ctx
      end function
      integer(c_int) function fwt_destroy(ctx) bind(C, name="fwt_destroy")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function fwt_load_inputs(ctx, cpath, ppath) bind(C, name="fwt_load_inputs")
         import :: c_int, c_ptr, c_char
         type(c_ptr), value :: ctx
         character(kind=c_char) :: cpath(*), ppath(*)
      end function
      integer(c_int) function fwt_set_centerlines(ctx, nline, npoint, xyz, sigma, gamma, n_t, if_filter) &
         bind(C, name="fwt_set_centerlines")
         import :: c_int, c_ptr, c_int64_t, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: nline
         integer(c_int64_t) :: npoint(*)
         real(c_double) :: xyz(*), sigma(*), gamma(*)
         integer(c_int) :: n_t(*), if_filter(*)
      end function
      ! the copy runs behind the deposition: xyz must stay allocated and unchanged until the
      ! next fwt_deposit / fwt_run returns
      integer(c_int) function fwt_set_centerlines_async(ctx, nline, npoint, xyz, sigma, gamma, n_t, if_filter) &
         bind(C, name="fwt_set_centerlines_async")
         import :: c_int, c_ptr, c_int64_t, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: nline
         integer(c_int64_t) :: npoint(*)
         real(c_double) :: xyz(*), sigma(*), gamma(*)
         integer(c_int) :: n_t(*), if_filter(*)
      end function
      integer(c_int) function fwt_deposit(ctx, line_s, line_e) bind(C, name="fwt_deposit")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: line_s, line_e
      end function
      integer(c_int) function fwt_biot_savart(ctx) bind(C, name="fwt_biot_savart")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function fwt_normalize(ctx, up, etot, enstrophy) bind(C, name="fwt_normalize")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         real(c_double) :: up, etot, enstrophy
      end function
      integer(c_int) function fwt_run(ctx) bind(C, name="fwt_run")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function fwt_write_outputs(ctx, outdir) bind(C, name="fwt_write_outputs")
         import :: c_int, c_ptr, c_char
         type(c_ptr), value :: ctx
         character(kind=c_char) :: outdir(*)
      end function
      integer(c_int) function fwt_copy_field(ctx, which, comp, host) bind(C, name="fwt_copy_field")
         import :: c_int, c_ptr, c_double
         type(c_ptr), value :: ctx
         integer(c_int), value :: which, comp
         real(c_double) :: host(*)
      end function
      integer(c_int) function fwt_last_error(buf, n) bind(C, name="fwt_last_error")
         import :: c_int, c_char
         character(kind=c_char) :: buf(*)
         integer(c_int), value :: n
      end function
      ! the reference's u_out / d_out switches (tube.f90:55): field_uw.dat / field_wd.dat
      integer(c_int) function fwt_set_outputs(ctx, u_out, d_out) bind(C, name="fwt_set_outputs")
         import :: c_int, c_ptr
         type(c_ptr), value :: ctx
         integer(c_int), value :: u_out, d_out
      end function
  end interface
end module fwt_iface
