! main.F90 -- Fortran 90 host driver of the B200 HPCCG library.
!
! Follows HPCCGmain of the reference (MPI/src/main.F90:77-135) on one rank:
! read nx ny nz from the command line, generate the matrix, print the
! problem, and run cg with max_iter = 150 and tolerance = 0 (:127-130).  The
! CSR comes from the library's host generator hpccg_generate_matrix, which is
! bit-exact with generate_matrix (MPI/src/SparseMatrix.F90:68-185), so this
! program needs none of the reference's modules; the cg call is the C-ABI's
! hpccg_gpu_cg (numerics.F90:41-162 on the GPU).  A maintainer who keeps the
! reference's own modules uses numerics_gpu.F90 instead (a `cg` with the
! reference's interface).
!
! NOT COMPILED HERE: no Fortran compiler exists in this image (or on the GPU
! box, which runs the same image).  driver/hpccg_main.cpp is the same program
! in C++ and is the one the tests run.  With gfortran:
!   make -C hpccg-f90_b200 fortran    ->  hpccg-f90_b200/HPCCG-B200-F90 nx ny nz
program HPCCGmain_gpu
    use iso_c_binding
    use hpccg_gpu
    implicit none

    integer, parameter :: dp = kind(0d0)
    integer, parameter :: print_freq = 15
    character(len=32) :: arg
    integer(c_int32_t) :: nx, ny, nz, nrow
    integer(c_int32_t), allocatable :: rowindex(:), colindex(:)
    real(c_double), allocatable :: values(:), x(:), b(:), xexact(:), hist(:)
    integer(c_int64_t) :: nnz
    type(c_ptr) :: ctx
    integer(c_int32_t) :: niters, max_iter
    real(c_double) :: normr, tolerance
    real(c_float) :: ms
    integer(c_int) :: ierr
    integer :: k

    if (command_argument_count() /= 3) then
        print *, 'USAGE: ./HPCCG <nx> <ny> <nz>'
        stop
    end if
    call get_command_argument(1, arg)
    read (arg, *) nx
    call get_command_argument(2, arg)
    read (arg, *) ny
    call get_command_argument(3, arg)
    read (arg, *) nz

    nrow = nx * ny * nz
    ! capacity 27 entries a row, as the reference allocates (SparseMatrix.F90:119-121)
    allocate(rowindex(nrow + 1), colindex(27 * nrow), values(27 * nrow))
    allocate(x(nrow), b(nrow), xexact(nrow))
    ierr = hpccg_generate_matrix(nx, ny, nz, rowindex, colindex, values, x, b, xexact, nnz)
    if (ierr /= HPCCG_OK) stop 'hpccg_generate_matrix failed'

    ! printInfo (main.F90:33-75); "Total nonzeroes" is the reference's 27*N count
    print *, "HPCCG Benchmark"
    print *, "Using double precision"
    print *, "Total size (N x N):", nrow
    print *, "Total nonzeroes:", 27 * nrow
    print *, "MPI disabled."
    print *, "OpenMP disabled."

    niters = 0
    normr = 0.0_dp
    max_iter = 150
    tolerance = 0.0_dp

    ierr = hpccg_gpu_create(nrow, nnz, rowindex, colindex, values, ctx)
    if (ierr /= HPCCG_OK) stop 'hpccg_gpu_create failed'
    allocate(hist(max_iter + 1))
    ierr = hpccg_gpu_cg(ctx, b, x, max_iter, tolerance, niters, normr, hist)
    if (ierr /= HPCCG_OK .and. ierr /= HPCCG_ERR_BREAKDOWN) stop 'hpccg_gpu_cg failed'

    print *, "Initial Residual = ", hist(1)
    do k = 1, niters
        if (MOD(k, print_freq) == 0 .or. k + 1 == max_iter) then
            print "(a,i5,tr2,a,e20.10)", 'ITER', k, 'Residual', hist(k + 1)
        end if
    end do
    ierr = hpccg_gpu_last_solve_ms(ctx, ms)
    print "(a,tr1,a,tr1,f12.6,tr1,a)", 'TIMER:', 'Total', real(ms, dp) / 1000.0_dp, 'sec'
    print *, "Difference between computed and exact = ", maxval(abs(x - xexact))

    call hpccg_gpu_destroy(ctx)
    deallocate(rowindex, colindex, values, x, b, xexact, hist)
end program HPCCGmain_gpu
