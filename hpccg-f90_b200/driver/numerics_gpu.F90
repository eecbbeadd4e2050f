! numerics_gpu.F90 -- the drop-in for the reference's `cg`
! (MPI/src/numerics.F90:41-162): same name, same arguments, same intents, same
! report lines, with the whole solve on the GPU through the C-ABI.
!
! A maintainer of the reference adds this file and hpccg_gpu.F90 to MPI/src,
! and in main.F90 replaces `use numerics` by `use numerics_gpu`; the call at
! MPI/src/main.F90:130 stays `call cg( A, b, x, max_iter, tolerance, niters,
! normr)`.  It uses the reference's own SparseMatrix module (SparseMatrixT,
! MPI/src/SparseMatrix.F90:44-64) and constants (dp).  exchange_externals is a
! no-op on one rank (MPI/src/SparseMatrix.F90:643-645) and is not called.
!
! NOT COMPILED HERE: no Fortran compiler in this image.  driver/main.F90 is a
! standalone program over the same interfaces; driver/hpccg_main.cpp is the
! tested C++ mirror.
module numerics_gpu
    use constants
    use iso_c_binding
    use hpccg_gpu
    implicit none
contains
    subroutine cg(A, b, x, max_iter, tolerance, niters, normr)
        use SparseMatrix
        implicit none
        type(SparseMatrixT), intent(inout) :: A
        real(kind=dp), allocatable, intent(inout) :: b(:)
        real(kind=dp), allocatable, intent(inout) :: x(:)
        integer, intent(in) :: max_iter
        real(kind=dp), intent(in) :: tolerance
        integer, intent(out) :: niters
        real(kind=dp), intent(out) :: normr

        integer, parameter :: print_freq = 15   ! as MPI/src/numerics.F90
        type(c_ptr) :: ctx
        real(c_double), allocatable :: hist(:)
        integer(c_int32_t) :: it
        real(c_double) :: nr
        real(c_float) :: ms
        integer(c_int) :: ierr
        integer :: k
        integer(c_int64_t) :: nnz

        nnz = int(A%rowindex(A%local_nrow + 1) - 1, c_int64_t)
        ierr = hpccg_gpu_create(int(A%local_nrow, c_int32_t), nnz, A%rowindex, A%colindex, &
                                A%values, ctx)
        if (ierr /= HPCCG_OK) stop 'hpccg_gpu_create failed'
        allocate(hist(max_iter + 1))
        ierr = hpccg_gpu_cg(ctx, b, x, int(max_iter, c_int32_t), real(tolerance, c_double), &
                            it, nr, hist)
        ! HPCCG_ERR_BREAKDOWN: the residual reached exactly 0 (tiny grids); x is
        ! the last finite iterate, where the reference would carry 0/0 on
        if (ierr /= HPCCG_OK .and. ierr /= HPCCG_ERR_BREAKDOWN) stop 'hpccg_gpu_cg failed'
        niters = it
        normr = nr

        print *, "Initial Residual = ", hist(1)
        do k = 1, niters
            if (MOD(k, print_freq) == 0 .or. k + 1 == max_iter) then
                print "(a,i5,tr2,a,e20.10)", 'ITER', k, 'Residual', hist(k + 1)
            end if
        end do
        if (niters < max_iter .and. ierr == HPCCG_OK) print *, "Converged Solution"
        ierr = hpccg_gpu_last_solve_ms(ctx, ms)
        print "(a,tr1,a,tr1,f12.6,tr1,a)", 'TIMER:', 'Total', real(ms, dp) / 1000.0_dp, 'sec'

        deallocate(hist)
        call hpccg_gpu_destroy(ctx)
    end subroutine cg
end module numerics_gpu
