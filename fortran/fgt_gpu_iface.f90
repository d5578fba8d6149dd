! Fortran interface of the B200 point FGT (libfgt_b200.so).
!
! A Fortran host keeps calling `call pfgt(...)` with the 24 reference
! arguments (src/pfgt/pfgt.f:6-10): link libfgt_b200.so instead of pfgt.o;
! its gfortran-mangled symbol pfgt_ takes every argument by reference.
! This module adds the status-returning variant and the status query.
module fgt_gpu_iface
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: FGT_OK = 0
  integer(c_int), parameter :: FGT_PREC_AUTO = 0, FGT_PREC_FP64 = 1, FGT_PREC_MIXED = 2

  interface
    ! int fgt_pfgt_c(const fgt_opts*, ...): opts = c_null_ptr for defaults
    integer(c_int) function fgt_pfgt_c(opts, nd, dim, delta, eps, iperiod, bs0, cen0, ns, &
        sources, ifcharge, charge, ifdipole, rnormal, dipstr, ifpgh, pot, grad, hess, nt, &
        targ, ifpghtarg, pottarg, gradtarg, hesstarg) bind(C, name="fgt_pfgt_c")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: opts
      integer(c_int), value :: nd, dim, iperiod, ns, ifcharge, ifdipole, ifpgh, nt, ifpghtarg
      real(c_double), value :: delta, eps
      real(c_double) :: bs0, cen0(*)
      real(c_double) :: sources(*), charge(*), rnormal(*), dipstr(*)
      real(c_double) :: pot(*), grad(*), hess(*), targ(*), pottarg(*), gradtarg(*), hesstarg(*)
    end function fgt_pfgt_c

    integer(c_int) function fgt_last_status() bind(C, name="fgt_last_status")
      import :: c_int
    end function fgt_last_status
  end interface
end module fgt_gpu_iface
