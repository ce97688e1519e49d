!> ISO_C_BINDING interface to the B200 linear-equation library (include/mfixgpu.h)
!> and a drop-in SOLVE_LIN_EQ with the dummy list of model/solve_lin_eq.f:17-78.
!>
!> Link this module and libmfixgpu.so in place of model/solve_lin_eq.f; every
!> caller (model/solve_vel_star.f:315, model/solve_pp_g.f:119, ...) is unchanged.
!> Call MFIXGPU_SETUP once after SET_INCREMENTS (it registers the box geometry
!> the library cannot read from the MFIX modules).
module mfixgpu_mod
   use iso_c_binding, only: c_int, c_int64_t, c_long_long, c_double, c_char, c_ptr, c_null_char, c_null_ptr, &
                            c_loc, c_size_t
   implicit none
   private
   public :: mfixgpu_setup, mfixgpu_set_option, mfixgpu_iter_tot, mfixgpu_finalize, mfixgpu_flush, &
             solve_lin_eq_defer, solve_pp_g_gpu

   !> mfixgpu_pp_fields (include/mfixgpu.h): the fields SOLVE_PP_G assembles from
   type, bind(C) :: pp_fields_t
      type(c_ptr) :: flag = c_null_ptr
      type(c_ptr) :: rop_ge = c_null_ptr, rop_gn = c_null_ptr, rop_gt = c_null_ptr
      type(c_ptr) :: ayz = c_null_ptr, axz = c_null_ptr, axy = c_null_ptr
      type(c_ptr) :: u_g = c_null_ptr, v_g = c_null_ptr, w_g = c_null_ptr
      type(c_ptr) :: rop_g = c_null_ptr, rop_go = c_null_ptr, vol = c_null_ptr, sum_r_g = c_null_ptr
      type(c_ptr) :: d_e = c_null_ptr, d_n = c_null_ptr, d_t = c_null_ptr
      integer(c_int) :: mmax = 0, ro_g0_defined = 1
      type(c_ptr) :: close_packed = c_null_ptr
      type(c_ptr) :: rop_se = c_null_ptr, rop_sn = c_null_ptr, rop_st = c_null_ptr
      type(c_ptr) :: u_s = c_null_ptr, v_s = c_null_ptr, w_s = c_null_ptr
      type(c_ptr) :: rop_s = c_null_ptr, rop_so = c_null_ptr, sum_r_s = c_null_ptr
      real(c_double) :: odt = 0
      integer(c_long_long) :: ijk_p_g = 0
      integer(c_int) :: on_device = 0, pad = 0
   end type pp_fields_t

   interface
      integer(c_int) function c_init_geometry(imax2, jmax2, kmax2, do_k, dimension_3, dimension_m) &
            bind(C, name="mfixgpu_init_geometry")
         import :: c_int, c_int64_t
         integer(c_int), intent(in) :: imax2, jmax2, kmax2, do_k
         integer(c_int64_t), intent(in) :: dimension_3
         integer(c_int), intent(in) :: dimension_m
      end function c_init_geometry

      integer(c_int) function c_init_cyclic(cyclic_x, cyclic_y, cyclic_z) bind(C, name="mfixgpu_init_cyclic")
         import :: c_int
         integer(c_int), intent(in) :: cyclic_x, cyclic_y, cyclic_z
      end function c_init_cyclic

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

      subroutine c_solve_pp_g(f, normg, pp_g, resg, itmax, method, sweep, tol, pc, ier, sweep_len, pc_len) &
            bind(C, name="mfixgpu_solve_pp_g_")
         import :: pp_fields_t, c_int, c_double, c_char, c_size_t
         type(pp_fields_t), intent(in) :: f
         real(c_double), intent(in) :: normg, tol
         real(c_double), dimension(*), intent(inout) :: pp_g
         real(c_double), intent(out) :: resg
         integer(c_int), intent(in) :: itmax, method
         character(kind=c_char), dimension(*), intent(in) :: sweep, pc
         integer(c_int), intent(inout) :: ier
         integer(c_size_t), value :: sweep_len, pc_len
      end subroutine c_solve_pp_g
   end interface

contains

   !> Registers IMAX2, JMAX2, KMAX2, DO_K, DIMENSION_3, DIMENSION_M and the cyclic
   !> axes (CYCLIC_X/Y/Z, model/geometry_mod.f; their increments wrap as
   !> model/set_increments.f:73-113 builds them).
   subroutine mfixgpu_setup(ier)
      use geometry, only: imax2, jmax2, kmax2, do_k, cyclic_x, cyclic_y, cyclic_z
      use param, only: dimension_3, dimension_m
      integer, intent(out) :: ier
      integer(c_int) :: dk
      dk = 0
      if (do_k) dk = 1
      ier = c_init_geometry(int(imax2, c_int), int(jmax2, c_int), int(kmax2, c_int), dk, &
                            int(dimension_3, c_int64_t), int(dimension_m, c_int))
      if (ier /= 0) return
      ier = c_init_cyclic(merge(1_c_int, 0_c_int, cyclic_x), merge(1_c_int, 0_c_int, cyclic_y), &
                          merge(1_c_int, 0_c_int, cyclic_z))
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

   !> SOLVE_PP_G(NORMG, RESG, IER) (model/solve_pp_g.f:10-118) on the device: the
   !> pressure-correction system is assembled there from the fields below and solved
   !> there; only the fields and PP_G cross the host link, and A_M/B_M are not used.
   !> For an incompressible run (RO_G0 defined) on a Cartesian grid without shear,
   !> point sources or user sources; other runs keep the reference's SOLVE_PP_G.
   !> The addresses of the module arrays are taken through TARGET dummies, so the
   !> arrays must be contiguous (they are: MFIX allocates them whole).
   subroutine solve_pp_g_gpu(normg, resg, ier)
      use fldvar, only: rop_g, rop_go, u_g, v_g, w_g, rop_s, rop_so, u_s, v_s, w_s
      use mflux, only: rop_ge, rop_gn, rop_gt, rop_se, rop_sn, rop_st
      use geometry, only: flag, ayz, axz, axy, vol, do_k
      use pgcor, only: pp_g, d_e, d_n, d_t
      use physprop, only: mmax, close_packed, ro_g0
      use rxns, only: sum_r_g, sum_r_s
      use run, only: odt
      use bc, only: ijk_p_g
      use param1, only: undefined, undefined_i
      use leqsol, only: leq_it, leq_method, leq_sweep, leq_tol, leq_pc
      double precision, intent(in) :: normg
      double precision, intent(out) :: resg
      integer, intent(inout) :: ier
      type(pp_fields_t) :: f
      integer(c_int), allocatable, target :: cp(:)
      integer(c_int) :: cier
      real(c_double) :: cres
      integer :: m
      f%flag = iaddr(flag)
      f%rop_ge = daddr(rop_ge); f%rop_gn = daddr(rop_gn)
      f%ayz = daddr(ayz); f%axz = daddr(axz)
      f%u_g = daddr(u_g); f%v_g = daddr(v_g)
      f%rop_g = daddr(rop_g); f%rop_go = daddr(rop_go); f%vol = daddr(vol); f%sum_r_g = daddr(sum_r_g)
      f%d_e = daddr(d_e); f%d_n = daddr(d_n)
      if (do_k) then
         f%rop_gt = daddr(rop_gt); f%axy = daddr(axy); f%w_g = daddr(w_g); f%d_t = daddr(d_t)
      end if
      f%mmax = int(mmax, c_int)
      allocate(cp(max(mmax, 1)))
      cp = 0
      do m = 1, mmax
         if (close_packed(m)) cp(m) = 1
      end do
      f%close_packed = c_loc(cp)
      if (mmax > 0) then
         f%rop_se = daddr(rop_se); f%rop_sn = daddr(rop_sn)
         f%u_s = daddr(u_s); f%v_s = daddr(v_s)
         f%rop_s = daddr(rop_s); f%rop_so = daddr(rop_so); f%sum_r_s = daddr(sum_r_s)
         if (do_k) then
            f%rop_st = daddr(rop_st); f%w_s = daddr(w_s)
         end if
      end if
      f%ro_g0_defined = merge(1_c_int, 0_c_int, ro_g0 /= undefined)
      f%odt = odt
      f%ijk_p_g = merge(int(ijk_p_g, c_long_long), 0_c_long_long, ijk_p_g /= undefined_i)
      cier = int(ier, c_int)
      call c_solve_pp_g(f, real(normg, c_double), pp_g, cres, int(leq_it(1), c_int), int(leq_method(1), c_int), &
                        leq_sweep(1), real(leq_tol(1), c_double), leq_pc(1), cier, 4_c_size_t, 4_c_size_t)
      resg = cres
      ier = int(cier)
      deallocate(cp)
   contains
      type(c_ptr) function daddr(x)
         double precision, target, intent(in) :: x(*)
         daddr = c_loc(x)
      end function daddr
      type(c_ptr) function iaddr(x)
         integer, target, intent(in) :: x(*)
         iaddr = c_loc(x)
      end function iaddr
   end subroutine solve_pp_g_gpu

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

