/*
 * hpccg_oracle.h -- CPU oracle for the HPCCG conjugate-gradient path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * Fortran 90 HPCCG (MPI/src, built sequentially: ENABLE_MPI=NO, ENABLE_OMP=NO)
 * used as the checker for the CUDA product and as the timed CPU baseline.
 * Nothing in the product links or calls it.
 *
 * Parity status: UNPINNED against reference outputs.  The reference ships no
 * tests, fixtures or golden vectors, and it is Fortran 90 with no Fortran
 * compiler available, so it cannot be run here.  The oracle is instead checked
 * against analytic known answers that follow from the reference's definitions:
 * nnz = (3nx-2)(3ny-2)(3nz-2), b = A*1 exactly, Initial Residual = ||b||,
 * x -> xexact = 1, and the row/column layout implied by the loop nest.
 *
 * Floating-point semantics: compiled with -O2 -ffp-contract=off (no FMA, no
 * reassociation), every loop runs in the reference's index order, so results
 * equal what gfortran -O2/-O3 (no -ffast-math) would give for MPI/src.
 * The OpenMP build (liboracle_omp.so) adds the reference's
 * "!$OMP PARALLEL DO [REDUCTION(+:)]" work sharing and is used for timing only.
 */
#ifndef HPCCG_ORACLE_H
#define HPCCG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* MPI/src/SparseMatrix.F90:68-185 generate_matrix, one rank.
 * rowindex: nrow+1 (1-based), colindex/values: 27*nrow (1-based cols),
 * x, b, xexact: nrow.  Returns the number of stored nonzeros. */
int64_t orc_generate_matrix(int32_t nx, int32_t ny, int32_t nz, int32_t *rowindex,
                            int32_t *colindex, double *values, double *x, double *b,
                            double *xexact);

/* MPI/src/SparseMatrix.F90:213-232 spmv: y(i) = sum_k values(k)*x(colindex(k)). */
void orc_spmv(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
              const double *values, const double *x, double *y);

/* Summation of orc_ddot/orc_ddot1: 0 = reference sequential order (default),
 * 1 = Neumaier-compensated (a near-exact value, to attribute differences). */
void orc_set_dot_mode(int mode);

/* MPI/src/vector_operations.F90:40-169 */
double orc_ddot(int32_t n, const double *x, const double *y);
double orc_ddot1(int32_t n, const double *x);
void orc_waxpby(int32_t n, double alpha, const double *x, double beta, const double *y,
                double *w);
void orc_wwpby(int32_t n, double beta, const double *y, double *w);
void orc_wxbw(int32_t n, const double *x, double beta, double *w);
void orc_vcopy(int32_t n, const double *x, double *y);

/* MPI/src/numerics.F90:41-162 cg.  x is updated in place.  hist (nullable,
 * length max_iter+1) receives hist[0] = Initial Residual and hist[k] = the
 * normr computed at iteration k (the value the reference prints), k=1..niters.
 * Returns 0. */
int orc_cg(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
           const double *values, const double *b, double *x, int32_t max_iter,
           double tolerance, int32_t *niters, double *normr, double *hist);

/* generate_matrix(nx,ny,nz)'s operator applied from the grid without storing
 * the CSR (MPI/src/SparseMatrix.F90:138-159 with spmv, :213-232): the same
 * terms in the same order, so y equals orc_spmv on the generated CSR bit for
 * bit.  For checks at sizes where the host CSR (12 bytes per nonzero) is
 * wasteful: 256^3 holds 5.4 GB of it. */
void orc_grid_spmv(int32_t nx, int32_t ny, int32_t nz, const double *x, double *y);
/* orc_cg with orc_grid_spmv as the operator (identical arithmetic). */
int orc_cg_grid(int32_t nx, int32_t ny, int32_t nz, const double *b, double *x,
                int32_t max_iter, double tolerance, int32_t *niters, double *normr,
                double *hist);
/* orc_true_relres with orc_grid_spmv as the operator. */
double orc_grid_true_relres(int32_t nx, int32_t ny, int32_t nz, const double *b,
                            const double *x);

/* orc_cg with caller-owned work arrays (work: 3*nrow doubles for r, p, Ap),
 * so that repeated timed solves neither allocate nor first-touch memory. */
int orc_cg_work(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
                const double *values, const double *b, double *x, int32_t max_iter,
                double tolerance, int32_t *niters, double *normr, double *hist,
                double *work);

/* MPI/src/numerics.F90:164-198 compute_residual: max_i |v1(i)-v2(i)|. */
double orc_compute_residual(int32_t n, const double *v1, const double *v2);

/* ||b - A x||_2 / ||b||_2 in sequential FP64 (the convergence criterion). */
double orc_true_relres(int32_t nrow, const int32_t *rowindex, const int32_t *colindex,
                       const double *values, const double *b, const double *x);

/* MPI/src/SparseMatrix.F90:68-185 on rank `rank` of `nranks`: the rows
 * local_nrow*rank+1 .. local_nrow*(rank+1) of the weak-scaled problem (the
 * nx x ny x (nz*nranks) grid cut into z slabs), with global 1-based columns.
 * orc_generate_matrix is rank 0 of 1. */
int64_t orc_generate_matrix_rank(int32_t nx, int32_t ny, int32_t nz, int32_t rank, int32_t nranks,
                                 int32_t *rowindex, int32_t *colindex, double *values, double *x,
                                 double *b, double *xexact);

/* The multi-rank halo set-up of every rank of an nranks communicator,
 * simulated in one process (hpccg_oracle_slab.c): mode 0 follows the MPI
 * variant's make_local_matrix (MPI/src/SparseMatrix.F90:235-627), mode 1 the
 * CAF-V2 variant's (CAF-V2/src/SparseMatrix.F90:205-331). */
typedef struct orc_slab_plan orc_slab_plan;
orc_slab_plan *orc_slab_plan_create(int32_t nx, int32_t ny, int32_t nz, int32_t nranks, int32_t mode);
void orc_slab_plan_destroy(orc_slab_plan *plan);
/* Copies one of a rank's lists into out (nullable) and returns its length.
 * Indices keep the reference's 1-based convention; ranks are 0-based. */
enum {
    ORC_SLAB_NNZ = 0,               /* (count only) stored nonzeros */
    ORC_SLAB_COLINDEX = 1,          /* local column indices after renumbering */
    ORC_SLAB_ROWINDEX = 2,
    ORC_SLAB_EXTERNALS = 3,         /* global id of each local external, in local order */
    ORC_SLAB_EXTERNAL_OWNERS = 4,   /* owning rank of each local external */
    ORC_SLAB_NEIGHBORS = 5,         /* mode 0: neighbours in receive order */
    ORC_SLAB_RECV_LENGTH = 6,       /* mode 0: block sizes */
    ORC_SLAB_RECV_LENGTH_LITERAL = 7, /* mode 0: the reference loop's count */
    ORC_SLAB_SEND_LENGTH = 8,       /* mode 0 */
    ORC_SLAB_ELEMENTS_TO_SEND = 9,  /* mode 0: local indices, neighbour by neighbour */
    ORC_SLAB_BLOCKS = 10,           /* mode 1: 4 per block: owner, start, inmin, inmax */
    ORC_SLAB_REMOTE_INDEX = 11      /* mode 1: owner-local index of each external */
};
int32_t orc_slab_plan_get(const orc_slab_plan *plan, int32_t rank, int32_t what, int32_t *out);
/* MPI/src/numerics.F90:41-162 on all ranks in step (exchange before each
 * spmv, dot products summed over ranks in rank order).  b, x: the ranks'
 * vectors one after another. */
int orc_cg_slabs(const orc_slab_plan *plan, const double *b, double *x, int32_t max_iter,
                 double tolerance, int32_t *niters, double *normr, double *hist);

/* The project's counter-based generator (no reference counterpart): value i of
 * stream `seed` is splitmix64's finaliser applied to seed + (i+1)*golden;
 * uniform in [-1,1) is 2*((z>>11)*2^-53) - 1. */
uint64_t orc_splitmix64_at(uint64_t seed, uint64_t i);
void orc_uniform_pm1(uint64_t seed, int64_t n, double *out);
/* Grid sizes for the batched workload: sizes[3*s+d] = lo + (z mod (hi-lo+1)),
 * z = orc_splitmix64_at(seed, 3*s+d). */
void orc_batch_sizes(uint64_t seed, int32_t nsys, int32_t lo, int32_t hi, int32_t *sizes);

#ifdef __cplusplus
}
#endif
#endif
