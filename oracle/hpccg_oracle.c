/*
 * hpccg_oracle.c -- CPU oracle for the HPCCG conjugate-gradient path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product and the timed
 * CPU baseline, never part of the product.  Parity status: UNPINNED against
 * reference outputs (the Fortran reference cannot be compiled here and ships
 * no golden vectors); checked against analytic known answers instead.
 * Each function cites the reference routine it restates (paths are within
 * the RRZE-HPC/HPCCG-F90 project, MPI variant, single rank).
 *
 * Build: see oracle/Makefile (-O2 -ffp-contract=off; OpenMP variant for timing).
 */
#include "hpccg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* MPI/src/SparseMatrix.F90:68-185 on rank `rank` of `nranks` (weak scaling in
 * z): local_nrow = nx*ny*nz (:108), total_nrow = local_nrow*nranks (:110),
 * start_row = local_nrow*rank + 1 (:112); columns are global and 1-based, and
 * the z truncation test curcol in [1,total_nrow] (:153) clips only at the
 * first plane of rank 0 and the last plane of the last rank.  Loop nest
 * iz -> iy -> ix (x fastest), stencil sz -> sy -> sx, so columns ascend
 * inside each row. */
int64_t orc_generate_matrix_rank(int32_t nx, int32_t ny, int32_t nz, int32_t rank, int32_t nranks,
                                 int32_t *rowindex, int32_t *colindex, double *values, double *x,
                                 double *b, double *xexact)
{
    const int32_t local_nrow = nx * ny * nz;
    const int32_t total_nrow = local_nrow * nranks;
    const int32_t start_row = local_nrow * rank + 1;
    int32_t cursor = 1, rowcursor = 1;
    for (int32_t iz = 1; iz <= nz; ++iz) {
        for (int32_t iy = 1; iy <= ny; ++iy) {
            for (int32_t ix = 1; ix <= nx; ++ix) {
                const int32_t curlocalrow = (iz - 1) * nx * ny + (iy - 1) * nx + (ix - 1);
                const int32_t currow = start_row + curlocalrow;
                int32_t nnzrow = 0;
                rowindex[rowcursor - 1] = cursor;
                for (int32_t sz = -1; sz <= 1; ++sz) {
                    for (int32_t sy = -1; sy <= 1; ++sy) {
                        for (int32_t sx = -1; sx <= 1; ++sx) {
                            const int32_t curcol = currow + sz * nx * ny + sy * nx + sx;
                            if ((ix + sx >= 1) && (ix + sx <= nx) && (iy + sy >= 1) &&
                                (iy + sy <= ny) && (curcol >= 1 && curcol <= total_nrow)) {
                                values[cursor - 1] = (curcol == currow) ? 27.0 : -1.0;
                                colindex[cursor - 1] = curcol;
                                ++cursor;
                                ++nnzrow;
                            }
                        }
                    }
                }
                ++rowcursor;
                x[curlocalrow] = 0.0;
                b[curlocalrow] = 27.0 - (double)(nnzrow - 1);
                xexact[curlocalrow] = 1.0;
            }
        }
    }
    rowindex[rowcursor - 1] = cursor;
    return (int64_t)cursor - 1;
}

/* One rank: start_row = 1, total_nrow = local_nrow. */
int64_t orc_generate_matrix(int32_t nx, int32_t ny, int32_t nz, int32_t *rowindex,
                            int32_t *colindex, double *values, double *x, double *b,
                            double *xexact)
{
    return orc_generate_matrix_rank(nx, ny, nz, 0, 1, rowindex, colindex, values, x, b, xexact);
}

/* MPI/src/SparseMatrix.F90:213-232: row sum from 0.0 in increasing k. */
void orc_spmv(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
              const double *values, const double *x, double *y)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t i = 0; i < nrow; ++i) {
        double rowsum = 0.0;
        for (int32_t k = rowindex[i] - 1; k < rowindex[i + 1] - 1; ++k)
            rowsum = rowsum + values[k] * x[colindex[k] - 1];
        y[i] = rowsum;
    }
}

/* Dot-product summation used by orc_ddot/orc_ddot1 (and so by orc_cg):
 * 0 = the reference's sequential loop (default), 1 = Neumaier-compensated
 * sequential sum, a near-exact value used only to attribute differences
 * between the GPU's reassociated sums and the reference's own rounding. */
static int g_dot_mode = 0;
void orc_set_dot_mode(int mode) { g_dot_mode = mode; }

static double dot_compensated(int32_t n, const double *x, const double *y)
{
    double s = 0.0, c = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double t = x[i] * y[i];
        const double u = s + t;
        if (fabs(s) >= fabs(t))
            c += (s - u) + t;
        else
            c += (t - u) + s;
        s = u;
    }
    return s + c;
}

/* MPI/src/vector_operations.F90:40-71 ddot (single rank: no allreduce). */
double orc_ddot(int32_t n, const double *x, const double *y)
{
    if (g_dot_mode == 1)
        return dot_compensated(n, x, y);
    double local_result = 0.0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+ : local_result)
#endif
    for (int32_t i = 0; i < n; ++i)
        local_result = local_result + x[i] * y[i];
    return local_result;
}

/* MPI/src/vector_operations.F90:73-103 ddot1. */
double orc_ddot1(int32_t n, const double *x)
{
    if (g_dot_mode == 1)
        return dot_compensated(n, x, x);
    double local_result = 0.0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+ : local_result)
#endif
    for (int32_t i = 0; i < n; ++i)
        local_result = local_result + x[i] * x[i];
    return local_result;
}

/* MPI/src/vector_operations.F90:105-121 waxpby: w = alpha*x + beta*y. */
void orc_waxpby(int32_t n, double alpha, const double *x, double beta, const double *y,
                double *w)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t i = 0; i < n; ++i)
        w[i] = alpha * x[i] + beta * y[i];
}

/* MPI/src/vector_operations.F90:123-137 wwpby: w = w + beta*y. */
void orc_wwpby(int32_t n, double beta, const double *y, double *w)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t i = 0; i < n; ++i)
        w[i] = w[i] + beta * y[i];
}

/* MPI/src/vector_operations.F90:139-153 wxbw: w = x + beta*w. */
void orc_wxbw(int32_t n, const double *x, double beta, double *w)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t i = 0; i < n; ++i)
        w[i] = x[i] + beta * w[i];
}

/* MPI/src/vector_operations.F90:155-169 vcopy: y = x. */
void orc_vcopy(int32_t n, const double *x, double *y)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t i = 0; i < n; ++i)
        y[i] = x[i];
}

/* generate_matrix's operator applied without storing it
 * (MPI/src/SparseMatrix.F90:138-159 fused with spmv, :213-232): row i sums, from
 * 0.0, value*x(col) over the stencil in the sz -> sy -> sx order the CSR stores,
 * with 27.0 on the diagonal and -1.0 elsewhere, skipping the neighbours the
 * generator drops.  The operations are those of orc_spmv on the generated CSR,
 * so y is bit-identical to it; only the 12 bytes per nonzero are not needed. */
void orc_grid_spmv(int32_t nx, int32_t ny, int32_t nz, const double *x, double *y)
{
    const int64_t nxy = (int64_t)nx * ny;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t iz = 0; iz < nz; ++iz) {
        for (int32_t iy = 0; iy < ny; ++iy) {
            for (int32_t ix = 0; ix < nx; ++ix) {
                const int64_t row = iz * nxy + (int64_t)iy * nx + ix;
                double rowsum = 0.0;
                for (int32_t sz = -1; sz <= 1; ++sz) {
                    if (iz + sz < 0 || iz + sz >= nz)
                        continue;
                    for (int32_t sy = -1; sy <= 1; ++sy) {
                        if (iy + sy < 0 || iy + sy >= ny)
                            continue;
                        for (int32_t sx = -1; sx <= 1; ++sx) {
                            if (ix + sx < 0 || ix + sx >= nx)
                                continue;
                            const int64_t col = row + sz * nxy + (int64_t)sy * nx + sx;
                            const double v = (col == row) ? 27.0 : -1.0;
                            rowsum = rowsum + v * x[col];
                        }
                    }
                }
                y[row] = rowsum;
            }
        }
    }
}

/* The operator orc_cg applies: a stored CSR or the generator's grid. */
typedef struct {
    int32_t nrow;
    const int32_t *rowindex, *colindex;
    const double *values;
    int32_t nx, ny, nz; /* grid operator when rowindex == NULL */
} orc_op;

static void op_apply(const orc_op *op, const double *x, double *y)
{
    if (op->rowindex)
        orc_spmv(op->nrow, op->rowindex, op->colindex, op->values, x, y);
    else
        orc_grid_spmv(op->nx, op->ny, op->nz, x, y);
}

/* MPI/src/numerics.F90:41-162 cg, single rank (exchange_externals is a no-op,
 * SparseMatrix.F90:643-645).  Operation order as in the reference:
 * prepare (:91-104), then per k (:108-147): stop test on the normr of the
 * previous iteration, k==1 vcopy else ddot1/beta/wxbw, normr = sqrt(rtrans),
 * spmv, ddot, alpha, r update before x update. */
static int cg_core(const orc_op *op, const double *b, double *x, int32_t max_iter,
                   double tolerance, int32_t *niters, double *normr_out, double *hist,
                   double *work)
{
    const int32_t nrow = op->nrow;
    /* r, p, Ap: the reference allocates them per call (numerics.F90:83-85);
     * a caller that times repeated solves may pass them in (3*nrow doubles) */
    double *r = work ? work : (double *)malloc(sizeof(double) * (size_t)nrow);
    double *p = work ? work + nrow : (double *)malloc(sizeof(double) * (size_t)nrow);
    double *Ap = work ? work + 2 * (size_t)nrow : (double *)malloc(sizeof(double) * (size_t)nrow);
    double normr = 0.0, rtrans = 0.0, oldrtrans = 0.0, alpha, beta;
    int32_t it = 0;

    orc_vcopy(nrow, x, p);
    op_apply(op, p, Ap);
    orc_waxpby(nrow, 1.0, b, -1.0, Ap, r);
    rtrans = orc_ddot1(nrow, r);
    normr = sqrt(rtrans);
    if (hist)
        hist[0] = normr;

    for (int32_t k = 1; k <= max_iter; ++k) {
        if (normr < tolerance)
            break;
        if (k == 1) {
            orc_vcopy(nrow, r, p);
        } else {
            oldrtrans = rtrans;
            rtrans = orc_ddot1(nrow, r);
            beta = rtrans / oldrtrans;
            orc_wxbw(nrow, r, beta, p);
        }
        normr = sqrt(rtrans);
        if (hist)
            hist[k] = normr;
        op_apply(op, p, Ap);
        alpha = orc_ddot(nrow, p, Ap);
        alpha = rtrans / alpha;
        orc_wwpby(nrow, -alpha, Ap, r);
        orc_wwpby(nrow, alpha, p, x);
        it = k;
    }
    *niters = it;
    *normr_out = normr;
    if (!work) {
        free(r);
        free(p);
        free(Ap);
    }
    return 0;
}

int orc_cg(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
           const double *values, const double *b, double *x, int32_t max_iter,
           double tolerance, int32_t *niters, double *normr_out, double *hist)
{
    const orc_op op = {nrow, rowindex, colindex, values, 0, 0, 0};
    return cg_core(&op, b, x, max_iter, tolerance, niters, normr_out, hist, NULL);
}

int orc_cg_work(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
                const double *values, const double *b, double *x, int32_t max_iter,
                double tolerance, int32_t *niters, double *normr_out, double *hist,
                double *work)
{
    const orc_op op = {nrow, rowindex, colindex, values, 0, 0, 0};
    return cg_core(&op, b, x, max_iter, tolerance, niters, normr_out, hist, work);
}

int orc_cg_grid(int32_t nx, int32_t ny, int32_t nz, const double *b, double *x,
                int32_t max_iter, double tolerance, int32_t *niters, double *normr_out,
                double *hist)
{
    const orc_op op = {nx * ny * nz, NULL, NULL, NULL, nx, ny, nz};
    return cg_core(&op, b, x, max_iter, tolerance, niters, normr_out, hist, NULL);
}

/* MPI/src/numerics.F90:164-198 compute_residual (max-norm of v1-v2). */
double orc_compute_residual(int32_t n, const double *v1, const double *v2)
{
    double local_residual = 0.0;
    for (int32_t i = 0; i < n; ++i) {
        const double diff = fabs(v1[i] - v2[i]);
        if (diff > local_residual)
            local_residual = diff;
    }
    return local_residual;
}

double orc_true_relres(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
                       const double *values, const double *b, const double *x)
{
    double *Ax = (double *)malloc(sizeof(double) * (size_t)nrow);
    orc_spmv(nrow, rowindex, colindex, values, x, Ax);
    double rr = 0.0, bb = 0.0;
    for (int32_t i = 0; i < nrow; ++i) {
        const double ri = b[i] - Ax[i];
        rr = rr + ri * ri;
        bb = bb + b[i] * b[i];
    }
    free(Ax);
    return sqrt(rr) / sqrt(bb);
}

double orc_grid_true_relres(int32_t nx, int32_t ny, int32_t nz, const double *b,
                            const double *x)
{
    const int32_t nrow = nx * ny * nz;
    double *Ax = (double *)malloc(sizeof(double) * (size_t)nrow);
    orc_grid_spmv(nx, ny, nz, x, Ax);
    double rr = 0.0, bb = 0.0;
    for (int32_t i = 0; i < nrow; ++i) {
        const double ri = b[i] - Ax[i];
        rr = rr + ri * ri;
        bb = bb + b[i] * b[i];
    }
    free(Ax);
    return sqrt(rr) / sqrt(bb);
}

uint64_t orc_splitmix64_at(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1u) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void orc_uniform_pm1(uint64_t seed, int64_t n, double *out)
{
    for (int64_t i = 0; i < n; ++i) {
        const double u = (double)(orc_splitmix64_at(seed, (uint64_t)i) >> 11) * 0x1.0p-53;
        out[i] = 2.0 * u - 1.0;
    }
}

void orc_batch_sizes(uint64_t seed, int32_t nsys, int32_t lo, int32_t hi, int32_t *sizes)
{
    const uint64_t span = (uint64_t)(hi - lo + 1);
    for (int32_t j = 0; j < 3 * nsys; ++j)
        sizes[j] = lo + (int32_t)(orc_splitmix64_at(seed, (uint64_t)j) % span);
}
