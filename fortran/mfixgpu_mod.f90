!> ISO_C_BINDING interface to the B200 linear-equation library (include/mfixgpu.h)
!> and a drop-in SOLVE_LIN_EQ with the dummy list of model/solve_lin_eq.f:17-78.
!>
!> Link this module and libmfixgpu.so in place of model/solve_lin_eq.f; every
!> caller (model/solve_vel_star.f:315, model/solve_pp_g.f:119, ...) is unchanged.
!> Call MFIXGPU_SETUP once after SET_INCREMENTS (it registers the box geometry
!> the library cannot read from the MFIX modules).
module mfixgpu_mod
   use iso_c_binding, only: c_int, c_int64_t, c_double, c_char, c_ptr, c_null_char
   implicit none
   private
   public :: mfixgpu_setup, mfixgpu_set_option, mfixgpu_iter_tot, mfixgpu_finalize, mfixgpu_flush, &
             solve_lin_eq_defer

   interface
      integer(c_int) function c_init_geometry(imax2, jmax2, kmax2, do_k, dimension_3, dimension_m) &
            bind(C, name="mfixgpu_init_geometry")
         import :: c_int, c_int64_t
         integer(c_int), intent(in) :: imax2, jmax2, kmax2, do_k
         integer(c_int64_t), intent(in) :: dimension_3
         integer(c_int), intent(in) :: dimension_m
      end function c_init_geometry

      subroutine c_solve_lin_eq(vname, vname_len, vno, var, a_m, b_m, m, itmax, method, &
            sweep, sweep_len, tol1, pc, pc_len, ier) bind(C, name="mfixgpu_solve_lin_eq")
         import :: c_int, c_double, c_char
         character(kind=c_char), dimension(*), intent(in) :: vname
         integer(c_int), value :: vname_len, vno, m, itmax, method, sweep_len, pc_len
         real(c_double), dimension(*), intent(inout) :: var, a_m, b_m
         character(kind=c_char), dimension(*), intent(in) :: sweep, pc
         real(c_double), value :: tol1
         integer(c_int), intent(inout) :: ier
      end subroutine c_solve_lin_eq

      integer(c_int) function c_set_option(name, value) bind(C, name="mfixgpu_set_option")
         import :: c_int, c_char, c_double
         character(kind=c_char), dimension(*), intent(in) :: name
         real(c_double), value :: value
      end function c_set_option

      integer(c_int) function c_iter_tot(vno) bind(C, name="mfixgpu_iter_tot")
         import :: c_int
         integer(c_int), value :: vno
      end function c_iter_tot

      subroutine c_finalize() bind(C, name="mfixgpu_finalize")
      end subroutine c_finalize

      integer(c_int) function c_flush() bind(C, name="mfixgpu_solve_lin_eq_flush")
         import :: c_int
      end function c_flush
   end interface

contains

   !> Registers IMAX2, JMAX2, KMAX2, DO_K, DIMENSION_3 and DIMENSION_M.
   subroutine mfixgpu_setup(ier)
      use geometry, only: imax2, jmax2, kmax2, do_k
      use param, only: dimension_3, dimension_m
      integer, intent(out) :: ier
      integer(c_int) :: dk
      dk = 0
      if (do_k) dk = 1
      ier = c_init_geometry(int(imax2, c_int), int(jmax2, c_int), int(kmax2, c_int), dk, &
                            int(dimension_3, c_int64_t), int(dimension_m, c_int))
   end subroutine mfixgpu_setup

   integer function mfixgpu_set_option(name, value)
      character(len=*), intent(in) :: name
      double precision, intent(in) :: value
      mfixgpu_set_option = c_set_option(trim(name)//c_null_char, real(value, c_double))
   end function mfixgpu_set_option

   integer function mfixgpu_iter_tot(vno)
      integer, intent(in) :: vno
      mfixgpu_iter_tot = c_iter_tot(int(vno, c_int))
   end function mfixgpu_iter_tot

   subroutine mfixgpu_finalize()
      call c_finalize()
   end subroutine mfixgpu_finalize

   !> Solves every call queued by SOLVE_LIN_EQ_DEFER as one batch and writes their
   !> IERs; returns 0 or the first error code.
   integer function mfixgpu_flush()
      mfixgpu_flush = c_flush()
   end function mfixgpu_flush

   !> SOLVE_LIN_EQ_DEFER: SOLVE_LIN_EQ's dummy list, the call queued for MFIXGPU_FLUSH
   !> (the per-phase calls of one equation, e.g. model/solve_vel_star.f:308-331, then
   !> solve as one batch).  The library keeps the addresses of VAR, A_M, B_M and IER
   !> and writes through them at the flush, after this call has returned, so:
   !>  * the dummies carry ASYNCHRONOUS, and the caller declares the actual arguments
   !>    ASYNCHRONOUS (or TARGET) in the scope that calls SOLVE_LIN_EQ_DEFER and
   !>    MFIXGPU_FLUSH, so that no value of them is kept in a register across the flush;
   !>  * VAR, A_M and B_M are whole contiguous arrays (no array sections: a section
   !>    would be passed as a copy that is gone by the flush; the explicit interface of
   !>    this module procedure makes the compiler refuse one);
   !>  * VAR, A_M, B_M and IER stay in place and untouched until the flush; IER reads
   !>    -15 until then.
   !> The library's entry point takes gfortran's implicit convention (every argument by
   !> reference, the CHARACTER lengths appended), so it is called without an interface.
   subroutine solve_lin_eq_defer(vname, vno, var, a_m, b_m, m, itmax, method, sweep, tol1, pc, ier)
      use param, only: dimension_3, dimension_m
      character(len=*), intent(in) :: vname
      integer, intent(in) :: vno
      double precision, intent(inout), asynchronous :: var(dimension_3)
      double precision, intent(inout), asynchronous :: a_m(dimension_3, -3:3, 0:dimension_m)
      double precision, intent(inout), asynchronous :: b_m(dimension_3, 0:dimension_m)
      integer, intent(in) :: m, itmax, method
      character(len=4), intent(in) :: sweep
      double precision, intent(in) :: tol1
      character(len=4), intent(in) :: pc
      integer, intent(inout), asynchronous :: ier
      external mfixgpu_solve_lin_eq_defer
      call mfixgpu_solve_lin_eq_defer(vname, vno, var, a_m, b_m, m, itmax, method, sweep, tol1, pc, ier)
   end subroutine solve_lin_eq_defer

end module mfixgpu_mod

!> SOLVE_LIN_EQ with the reference's dummy list (model/solve_lin_eq.f:17-78):
!> A_M and B_M are the whole arrays, M selects the phase, exactly as the callers
!> pass them.  IER follows model/leq_bicgs.f; codes <= -10 are the library's
!> (include/mfixgpu.h) where the reference would stop the run.
subroutine solve_lin_eq(vname, vno, var, a_m, b_m, m, itmax, method, sweep, tol1, pc, ier)
   use iso_c_binding, only: c_int, c_double
   use param, only: dimension_3, dimension_m
   implicit none
   character(len=*), intent(in) :: vname
   integer, intent(in) :: vno
   double precision, intent(inout) :: var(dimension_3)
   double precision, intent(inout) :: a_m(dimension_3, -3:3, 0:dimension_m)
   double precision, intent(inout) :: b_m(dimension_3, 0:dimension_m)
   integer, intent(in) :: m, itmax, method
   character(len=4), intent(in) :: sweep
   double precision, intent(in) :: tol1
   character(len=4), intent(in) :: pc
   integer, intent(inout) :: ier
   interface
      subroutine c_solve_lin_eq(vname, vname_len, vno, var, a_m, b_m, m, itmax, method, &
            sweep, sweep_len, tol1, pc, pc_len, ier) bind(C, name="mfixgpu_solve_lin_eq")
         import :: c_int, c_double
         character(len=1), dimension(*), intent(in) :: vname
         integer(c_int), value :: vname_len, vno, m, itmax, method, sweep_len, pc_len
         real(c_double), dimension(*), intent(inout) :: var, a_m, b_m
         character(len=1), dimension(*), intent(in) :: sweep, pc
         real(c_double), value :: tol1
         integer(c_int), intent(inout) :: ier
      end subroutine c_solve_lin_eq
   end interface
   integer(c_int) :: cier
   cier = int(ier, c_int)
   call c_solve_lin_eq(vname, int(len(vname), c_int), int(vno, c_int), var, a_m, b_m, int(m, c_int), &
                       int(itmax, c_int), int(method, c_int), sweep, 4_c_int, real(tol1, c_double), pc, 4_c_int, cier)
   ier = int(cier)
end subroutine solve_lin_eq

