!==============================================================================!
  module Tf_Krylov_Mod
!------------------------------------------------------------------------------!
!>  ISO_C_BINDING interface to libtfkrylov.so, the B200 implementation of
!>  Native_Mod's Cg/Bicg (include/tf_krylov.h).  Solve_Native keeps its
!>  argument list; its body calls Tf_Solve below instead of Nat % Cg /
!>  Nat % Bicg.  Matrix_Type (Matrix_Mod.f90:57-76) gains one component,
!>      type(c_ptr) :: dev = c_null_ptr   ! device copy of row/col/dia
!>  which Tf_Register sets once after Create_Matrix, so Solve_Native finds
!>  the registration of whichever matrix (Nat % A or Nat % M) it is given.
!>  Not compiled: neither the machine this was written on nor the GPU
!>  machines it was tested on have a Fortran compiler.
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

  contains

  !============================================================================!
  subroutine Tf_Register(A, n_cells, n_own)
  !----------------------------------------------------------------------------!
  !>  Uploads the structure of one Matrix_Type once (after Create_Matrix) and
  !>  keeps the handle in A % dev.
  !----------------------------------------------------------------------------!
    use Matrix_Mod
    type(Matrix_Type), intent(inout) :: A
    integer,           intent(in)    :: n_cells, n_own
    integer(c_int)     :: st
    integer(c_int64_t) :: nnz

    if(.not. c_associated(tf_ctx)) then
      st = tf_ctx_create(-1_c_int, tf_ctx)
      if(st .ne. TF_OK) stop 'tf_ctx_create failed'
    end if
    nnz = int(A % row(n_cells + 1) - 1, c_int64_t)
    st = tf_matrix_register(tf_ctx, int(n_cells, c_int), int(n_own, c_int),  &
                            nnz, A % row, A % col, A % dia, A % dev)
    if(st .ne. TF_OK) stop 'tf_matrix_register failed'
  end subroutine

  !============================================================================!
  integer function Tf_Solve(solver, prec, A, x, b, miter, niter, tol,  &
                            fin_res, norm)
  !----------------------------------------------------------------------------!
  !>  Solve_Native's arguments (Solve_Native.f90:2-27) in, the library's
  !>  status out (0, or 64 for an unknown solver as Solve_Native.f90:38).
  !>  x is x(-nb:n) as Solve_Native declares it; the library reads and
  !>  writes x(1:n) only.  An absent norm stays absent.
  !----------------------------------------------------------------------------!
    use Matrix_Mod
    character(*),      intent(in)    :: solver, prec
    type(Matrix_Type), intent(inout) :: A
    real,              intent(inout) :: x(:)      ! x(1:n) of Solve_Native's x
    real,              intent(inout) :: b(:)
    integer,           intent(in)    :: miter
    integer,           intent(out)   :: niter
    real,              intent(in)    :: tol
    real,              intent(out)   :: fin_res
    real,    optional, intent(in)    :: norm
    integer(c_int) :: it
    real(c_double) :: res

    Tf_Solve = tf_solve_native(tf_ctx, A % dev,                           &
                               trim(solver)//c_null_char,                 &
                               trim(prec)//c_null_char,                   &
                               A % val, x, b, int(miter, c_int), it,      &
                               real(tol, c_double), res, norm)
    niter   = it
    fin_res = res
  end function

  end module
