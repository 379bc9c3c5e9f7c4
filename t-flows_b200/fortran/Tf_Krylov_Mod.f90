!==============================================================================!
  module Tf_Krylov_Mod
!------------------------------------------------------------------------------!
!>  ISO_C_BINDING interface to libtfkrylov.so, the B200 implementation of
!>  Native_Mod's Cg/Bicg (include/tf_krylov.h).  Solve_Native keeps its
!>  argument list; its body calls Tf_Solve_Native_Gpu below instead of
!>  Nat % Cg / Nat % Bicg.  Not compiled in this repository (no Fortran
!>  compiler is available where it was written); see INTEGRATION.md.
!------------------------------------------------------------------------------!
  use iso_c_binding
!------------------------------------------------------------------------------!
  implicit none
!==============================================================================!

  integer(c_int), parameter :: TF_OK = 0

  interface

    integer(c_int) function tf_ctx_create(device, ctx)  &
                            bind(C, name='tf_ctx_create')
      import :: c_int, c_ptr
      integer(c_int), value :: device
      type(c_ptr)           :: ctx
    end function

    integer(c_int) function tf_matrix_register(ctx, n_cells, n_own, nnz,  &
                                               row, col, dia, mat)        &
                            bind(C, name='tf_matrix_register')
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr),        value :: ctx
      integer(c_int),     value :: n_cells, n_own
      integer(c_int64_t), value :: nnz
      integer(c_int)            :: row(*), col(*), dia(*)
      type(c_ptr)               :: mat
    end function

    ! norm is OPTIONAL: an absent optional reaches C as a null pointer
    ! (Fortran 2018, 18.3.6), which tf_solve_native reads as "absent".
    integer(c_int) function tf_solve_native(ctx, mat, solver, prec, val,  &
                                            x, b, miter, niter, tol,      &
                                            fin_res, norm)                &
                            bind(C, name='tf_solve_native')
      import :: c_int, c_double, c_ptr, c_char
      type(c_ptr),        value    :: ctx, mat
      character(c_char)            :: solver(*), prec(*)
      real(c_double)               :: val(*), x(*), b(*)
      integer(c_int),     value    :: miter
      integer(c_int)               :: niter
      real(c_double),     value    :: tol
      real(c_double)               :: fin_res
      real(c_double),     optional :: norm
    end function

    integer(c_int) function tf_host_pin(ptr, bytes)  &
                            bind(C, name='tf_host_pin')
      import :: c_int, c_ptr, c_size_t
      type(c_ptr),       value :: ptr
      integer(c_size_t), value :: bytes
    end function

  end interface

  type(c_ptr), save :: tf_ctx = c_null_ptr
  type(c_ptr), save :: tf_mat_a = c_null_ptr   ! Nat % A
  type(c_ptr), save :: tf_mat_m = c_null_ptr   ! Nat % M

  contains

  !============================================================================!
  subroutine Tf_Register(A, n_cells, n_own, mat)
  !----------------------------------------------------------------------------!
  !>  Uploads the structure of one Matrix_Type once (after Create_Matrix).
  !----------------------------------------------------------------------------!
    use Matrix_Mod
    type(Matrix_Type), intent(in)    :: A
    integer,           intent(in)    :: n_cells, n_own
    type(c_ptr),       intent(inout) :: mat
    integer(c_int) :: st
    integer(c_int64_t) :: nnz

    if(.not. c_associated(tf_ctx)) then
      st = tf_ctx_create(-1_c_int, tf_ctx)
      if(st .ne. TF_OK) stop 'tf_ctx_create failed'
    end if
    nnz = int(A % row(n_cells + 1) - 1, c_int64_t)
    st = tf_matrix_register(tf_ctx, int(n_cells, c_int), int(n_own, c_int),  &
                            nnz, A % row, A % col, A % dia, mat)
    if(st .ne. TF_OK) stop 'tf_matrix_register failed'
  end subroutine

  end module
