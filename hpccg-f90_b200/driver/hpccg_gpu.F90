! hpccg_gpu.F90 -- ISO_C_BINDING interfaces to the B200 HPCCG library
! (include/hpccg_gpu.h), for the Fortran 90 host.
!
! NOT COMPILED HERE: this image has no Fortran compiler (gfortran, ifort,
! flang and nvfortran are all absent, on this machine and on the GPU box).
! The tested host over the same C-ABI is driver/hpccg_main.cpp.  With a
! Fortran compiler:  gfortran -c hpccg_gpu.F90  (see `make fortran`).
!
! Argument conventions: arrays go through assumed-size dummies (x(*)), so an
! `allocatable` array of the caller (the reference's b, x, A%rowindex, ...,
! MPI/src/SparseMatrix.F90:44-64, MPI/src/numerics.F90:41-53) passes its
! storage directly; scalars the C side takes by value carry `value`; a
! hpccg_ctx* is a type(c_ptr).  Every function returns 0 (HPCCG_OK) or an
! HPCCG_ERR_* code.
module hpccg_gpu
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: HPCCG_OK = 0
    integer(c_int), parameter :: HPCCG_ERR_BREAKDOWN = 4
    integer(c_int), parameter :: HPCCG_ERR_NOT_CONVERGED = 6
    integer(c_int32_t), parameter :: HPCCG_SPMV_AUTO = 0
    integer(c_int32_t), parameter :: HPCCG_SPMV_STENCIL = 4
    integer(c_int32_t), parameter :: HPCCG_PREC_FP32 = 1
    integer(c_int32_t), parameter :: HPCCG_PREC_BF16 = 2

    type, bind(C) :: hpccg_mixed_info
        integer(c_int32_t) :: outer_iters
        integer(c_int32_t) :: inner_iters
        real(c_double) :: relres
        integer(c_int32_t) :: status
        integer(c_int32_t) :: reserved
    end type hpccg_mixed_info

    interface
        ! MPI/src/SparseMatrix.F90:68-185 generate_matrix, on the host, bit-exact.
        ! rowindex(nrow+1), colindex/values capacity 27*nrow, x/b/xexact(nrow).
        integer(c_int) function hpccg_generate_matrix(nx, ny, nz, rowindex, colindex, values, &
                                                      x, b, xexact, nnz) &
                bind(C, name="hpccg_generate_matrix")
            import :: c_int, c_int32_t, c_int64_t, c_double
            integer(c_int32_t), value :: nx, ny, nz
            integer(c_int32_t), intent(out) :: rowindex(*), colindex(*)
            real(c_double), intent(out) :: values(*), x(*), b(*), xexact(*)
            integer(c_int64_t), intent(out) :: nnz
        end function

        ! Uploads the reference's 1-based CSR (the matrix half of cg's A).
        integer(c_int) function hpccg_gpu_create(nrow, nnz, rowindex, colindex, values, ctx) &
                bind(C, name="hpccg_gpu_create")
            import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
            integer(c_int32_t), value :: nrow
            integer(c_int64_t), value :: nnz
            integer(c_int32_t), intent(in) :: rowindex(*), colindex(*)
            real(c_double), intent(in) :: values(*)
            type(c_ptr), intent(out) :: ctx
        end function

        ! MPI/src/numerics.F90:41-162 cg on host arrays; hist(max_iter+1) receives
        ! the Initial Residual and the normr of every iteration.
        integer(c_int) function hpccg_gpu_cg(ctx, b, x, max_iter, tolerance, niters, normr, hist) &
                bind(C, name="hpccg_gpu_cg")
            import :: c_int, c_int32_t, c_double, c_ptr
            type(c_ptr), value :: ctx
            real(c_double), intent(in) :: b(*)
            real(c_double), intent(inout) :: x(*)
            integer(c_int32_t), value :: max_iter
            real(c_double), value :: tolerance
            integer(c_int32_t), intent(out) :: niters
            real(c_double), intent(out) :: normr
            real(c_double), intent(out) :: hist(*)
        end function

        ! FP64 iterative refinement around an FP32 or BF16-value inner CG, to
        ! ||b - A x|| <= rel_tol ||b|| (FP64 true residual).
        integer(c_int) function hpccg_gpu_solve_mixed(ctx, b, x, precision, rel_tol, max_outer, &
                                                      max_inner, inner_rtol, info) &
                bind(C, name="hpccg_gpu_solve_mixed")
            import :: c_int, c_int32_t, c_double, c_ptr, hpccg_mixed_info
            type(c_ptr), value :: ctx
            real(c_double), intent(in) :: b(*)
            real(c_double), intent(inout) :: x(*)
            integer(c_int32_t), value :: precision, max_outer, max_inner
            real(c_double), value :: rel_tol, inner_rtol
            type(hpccg_mixed_info), intent(out) :: info
        end function

        ! Device check that A is generate_matrix(nx,ny,nz); enables the
        ! matrix-free SpMV (bit-identical results).
        integer(c_int) function hpccg_gpu_set_geometry(ctx, nx, ny, nz) &
                bind(C, name="hpccg_gpu_set_geometry")
            import :: c_int, c_int32_t, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: nx, ny, nz
        end function

        integer(c_int) function hpccg_gpu_set_spmv(ctx, kind, param) bind(C, name="hpccg_gpu_set_spmv")
            import :: c_int, c_int32_t, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: kind, param
        end function

        ! Device ms of the last hpccg_gpu_cg (CUDA events around the graph launch).
        integer(c_int) function hpccg_gpu_last_solve_ms(ctx, ms) bind(C, name="hpccg_gpu_last_solve_ms")
            import :: c_int, c_float, c_ptr
            type(c_ptr), value :: ctx
            real(c_float), intent(out) :: ms
        end function

        subroutine hpccg_gpu_destroy(ctx) bind(C, name="hpccg_gpu_destroy")
            import :: c_ptr
            type(c_ptr), value :: ctx
        end subroutine
    end interface
end module hpccg_gpu
