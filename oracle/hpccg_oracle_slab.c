/*
 * hpccg_oracle_slab.c -- CPU oracle for the multi-rank (z-slab) HPCCG path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the library's z-slab CG and its
 * halo plans, never part of the product.  Parity status: unpinned against
 * reference outputs, like the rest of the oracle (the Fortran reference
 * cannot be compiled here); the global matrix it builds is checked against
 * the single-rank generate_matrix on the stacked grid.
 *
 * All ranks of a communicator are simulated in one process.  Each rank's
 * data follows the reference routine cited beside it (paths within the
 * RRZE-HPC/HPCCG-F90 project):
 *   - the rank's rows: MPI/src/SparseMatrix.F90:68-185 (orc_generate_matrix_rank);
 *   - mode 0, the MPI variant: make_local_matrix, MPI/src/SparseMatrix.F90:235-627,
 *     and exchange_externals, :630-680;
 *   - mode 1, the CAF-V2 variant: make_local_matrix, CAF-V2/src/SparseMatrix.F90:205-331,
 *     and exchange_externals (one contiguous get per block), :333-370;
 *   - cg with the exchange before each spmv and the dot products summed over
 *     ranks: MPI/src/numerics.F90:41-162, MPI/src/vector_operations.F90:40-103
 *     (MPI_ALLREDUCE), CAF-V2/src/caf_collectives.F90:37-60 (CAF_CO_SUM: image 1
 *     adds the images' values in image order).  Both sums are taken here as
 *     the left fold over ranks in rank order.
 *
 * One deliberate difference from the MPI variant.  make_local_matrix's loop
 * that measures each neighbour's block of externals (:533-545, repeated at
 * :575-583) leaves early only when j reaches num_external and then adds one,
 * so its recv_length / length come out one too large for every block except
 * the last (and for a last block of one element).  With two ranks every rank
 * has one neighbour and the counts are right; with three or more the middle
 * ranks' halos would be shifted by one element.  The oracle keeps the literal
 * count (recv_length_literal, for the tests that document this) and uses the
 * block sizes themselves for the exchange, as the routine intends.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "hpccg_oracle.h"

typedef struct {
    int32_t local_nrow, start_row, stop_row, num_external, local_ncol;
    int64_t nnz;
    int32_t *rowindex, *colindex; /* colindex: local, 1-based (externals > local_nrow) */
    double *values;
    int32_t *external_index;     /* global id of local external i (1-based i) */
    int32_t *external_processor; /* owning rank (0-based) of local external i */
    /* mode 0 */
    int32_t num_neighbors;
    int32_t *neighbors, *recv_length, *recv_length_literal, *send_length;
    int32_t total_to_be_sent;
    int32_t *elements_to_send; /* local, 1-based */
    /* mode 1 */
    int32_t num_blocks;
    int32_t *blk_image, *blk_start, *blk_inmin, *blk_inmax; /* image 0-based; start 1-based */
    int32_t *remote_index;                                  /* 1-based local index on the owner */
} slab_rank;

struct orc_slab_plan {
    int32_t nx, ny, nz, nranks, mode;
    slab_rank *r;
};

static int32_t *ialloc(int64_t n) { return (int32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t)); }

/* MPI/src/SparseMatrix.F90:235-627, the part each rank computes alone:
 * renumbering, externals grouped by owner, neighbour list and block lengths. */
static void local_part_mpi(slab_rank *R, int32_t nranks, const int32_t *offsets, int32_t total_nrow)
{
    int32_t *externals = ialloc((int64_t)total_nrow + 1);
    int32_t *external_index = ialloc(R->nnz + 1);
    for (int32_t i = 0; i <= total_nrow; ++i)
        externals[i] = -1;
    int32_t num_external = 1;
    for (int32_t i = 1; i <= R->local_nrow; ++i) {
        for (int32_t j = R->rowindex[i - 1]; j <= R->rowindex[i] - 1; ++j) {
            const int32_t cur = R->colindex[j - 1];
            if (R->start_row <= cur && cur <= R->stop_row) {
                R->colindex[j - 1] = cur - R->start_row + 1;
            } else {
                if (externals[cur] == -1) {
                    externals[cur] = num_external;
                    num_external = num_external + 1;
                    external_index[num_external - 1] = cur;
                }
                R->colindex[j - 1] = -cur;
            }
        }
    }
    num_external = num_external - 1;
    /* owner: the last rank whose first row is <= the index (:330-343) */
    int32_t *external_processor = ialloc(num_external + 1);
    for (int32_t i = 1; i <= num_external; ++i) {
        for (int32_t j = nranks; j >= 1; --j) {
            if (offsets[j - 1] <= external_index[i]) {
                external_processor[i] = j;
                break;
            }
        }
    }
    /* consecutive local numbers for the externals of one owner (:349-364) */
    int32_t *external_local_index = ialloc(num_external + 1);
    for (int32_t i = 1; i <= num_external; ++i)
        external_local_index[i] = -1;
    int32_t counter = R->local_nrow + 1;
    for (int32_t i = 1; i <= num_external; ++i) {
        if (external_local_index[i] == -1) {
            external_local_index[i] = counter++;
            for (int32_t j = i + 1; j <= num_external; ++j)
                if (external_processor[j] == external_processor[i])
                    external_local_index[j] = counter++;
        }
    }
    for (int32_t i = 1; i <= R->local_nrow; ++i)
        for (int32_t j = R->rowindex[i - 1]; j <= R->rowindex[i] - 1; ++j)
            if (R->colindex[j - 1] < 0)
                R->colindex[j - 1] = external_local_index[externals[-R->colindex[j - 1]]];
    R->num_external = num_external;
    R->local_ncol = R->local_nrow + num_external;
    R->external_index = ialloc(num_external + 1);
    R->external_processor = ialloc(num_external + 1);
    for (int32_t i = 1; i <= num_external; ++i) {
        const int32_t k = external_local_index[i] - R->local_nrow;
        R->external_index[k] = external_index[i];     /* new_external (:512-514) */
        R->external_processor[k] = external_processor[i] - 1; /* new_external_processor, 0-based */
    }
    /* recv_list: owners in the order their blocks appear (:452-462) */
    R->neighbors = ialloc(nranks);
    R->recv_length = ialloc(nranks);
    R->recv_length_literal = ialloc(nranks);
    R->send_length = ialloc(nranks);
    R->num_neighbors = 0;
    for (int32_t i = 1; i <= num_external; ++i)
        if (i == 1 || R->external_processor[i - 1] != R->external_processor[i])
            R->neighbors[R->num_neighbors++] = R->external_processor[i];
    /* block lengths: the literal loop of :533-545 and the true block sizes */
    int32_t j = 1;
    for (int32_t i = 0; i < R->num_neighbors; ++i) {
        int32_t newlength = 0;
        while (j <= num_external && R->external_processor[j] == R->neighbors[i]) {
            newlength = newlength + 1;
            j = j + 1;
            if (j == num_external)
                break;
        }
        R->recv_length_literal[i] = newlength + 1;
    }
    for (int32_t i = 0; i < R->num_neighbors; ++i) {
        int32_t n = 0;
        for (int32_t k = 1; k <= num_external; ++k)
            n += R->external_processor[k] == R->neighbors[i];
        R->recv_length[i] = n;
    }
    free(externals);
    free(external_index);
    free(external_processor);
    free(external_local_index);
}

/* MPI/src/SparseMatrix.F90:563-610: each neighbour sends the global ids it
 * wants from this rank (its block of new_external); this rank stores them as
 * local indices in elements_to_send, in its neighbour order. */
static void send_part_mpi(struct orc_slab_plan *P, int32_t rank)
{
    slab_rank *R = &P->r[rank];
    int64_t total = 0;
    for (int32_t i = 0; i < R->num_neighbors; ++i) {
        const slab_rank *N = &P->r[R->neighbors[i]];
        int32_t n = 0;
        for (int32_t k = 1; k <= N->num_external; ++k)
            n += N->external_processor[k] == rank;
        R->send_length[i] = n;
        total += n;
    }
    R->total_to_be_sent = (int32_t)total;
    R->elements_to_send = ialloc(total + 1);
    int32_t pos = 1;
    for (int32_t i = 0; i < R->num_neighbors; ++i) {
        const slab_rank *N = &P->r[R->neighbors[i]];
        for (int32_t k = 1; k <= N->num_external; ++k)
            if (N->external_processor[k] == rank)
                R->elements_to_send[pos++] = N->external_index[k] - R->start_row + 1;
    }
}

/* CAF-V2/src/SparseMatrix.F90:205-331: externals keep their order of first
 * appearance; runs of externals with one owner form blocks, each with the
 * range [inmin, inmax] of owner-local indices it needs. */
static void local_part_get(slab_rank *R, int32_t nranks, int32_t total_nrow)
{
    int32_t *externals = ialloc((int64_t)total_nrow + 1);
    int32_t *external_index = ialloc(R->nnz + 1);
    const int32_t cap = (int32_t)R->nnz + 2;
    R->blk_image = ialloc(cap);
    R->blk_start = ialloc(cap + 1);
    R->blk_inmin = ialloc(cap);
    R->blk_inmax = ialloc(cap);
    for (int32_t i = 0; i <= total_nrow; ++i)
        externals[i] = -1;
    int32_t num_external = 1, num_blocks = 1;
    int32_t *image = R->blk_image; /* 1-based image numbers while scanning */
    image[1] = 0;
    R->blk_inmin[1] = 0x7fffffff;
    R->blk_inmax[1] = 0;
    for (int32_t i = 1; i <= R->local_nrow; ++i) {
        for (int32_t j = R->rowindex[i - 1]; j <= R->rowindex[i] - 1; ++j) {
            const int32_t cur = R->colindex[j - 1];
            if (R->start_row <= cur && cur <= R->stop_row) {
                R->colindex[j - 1] = cur - R->start_row + 1;
            } else {
                if (externals[cur] == -1) {
                    externals[cur] = num_external;
                    const int32_t img = (cur - 1) / R->local_nrow + 1;
                    if (image[num_blocks] == 0) {
                        image[num_blocks] = img;
                        R->blk_start[num_blocks] = num_external;
                    }
                    if (img != image[num_blocks]) {
                        num_blocks = num_blocks + 1;
                        image[num_blocks] = img;
                        R->blk_start[num_blocks] = num_external;
                        R->blk_inmin[num_blocks] = 0x7fffffff;
                        R->blk_inmax[num_blocks] = 0;
                    }
                    const int32_t ind = (cur - 1) % R->local_nrow + 1;
                    if (ind < R->blk_inmin[num_blocks])
                        R->blk_inmin[num_blocks] = ind;
                    if (ind > R->blk_inmax[num_blocks])
                        R->blk_inmax[num_blocks] = ind;
                    num_external = num_external + 1;
                    external_index[num_external - 1] = cur;
                }
                R->colindex[j - 1] = -cur;
            }
        }
    }
    R->blk_start[num_blocks + 1] = num_external;
    R->num_external = num_external - 1;
    R->num_blocks = nranks == 1 || R->num_external == 0 ? 0 : num_blocks;
    R->remote_index = ialloc(R->num_external + 1);
    R->external_index = ialloc(R->num_external + 1);
    R->external_processor = ialloc(R->num_external + 1);
    for (int32_t i = 1; i <= R->num_external; ++i) {
        R->remote_index[i] = (external_index[i] - 1) % R->local_nrow + 1;
        R->external_index[i] = external_index[i];
        R->external_processor[i] = (external_index[i] - 1) / R->local_nrow;
    }
    for (int32_t k = 1; k <= num_blocks; ++k)
        image[k] -= 1; /* 0-based ranks from here on */
    for (int32_t i = 1; i <= R->local_nrow; ++i)
        for (int32_t j = R->rowindex[i - 1]; j <= R->rowindex[i] - 1; ++j)
            if (R->colindex[j - 1] < 0)
                R->colindex[j - 1] = R->local_nrow + externals[-R->colindex[j - 1]];
    R->local_ncol = R->local_nrow + R->num_external;
    free(externals);
    free(external_index);
}

orc_slab_plan *orc_slab_plan_create(int32_t nx, int32_t ny, int32_t nz, int32_t nranks, int32_t mode)
{
    orc_slab_plan *P = (orc_slab_plan *)calloc(1, sizeof(orc_slab_plan));
    P->nx = nx, P->ny = ny, P->nz = nz, P->nranks = nranks, P->mode = mode;
    P->r = (slab_rank *)calloc((size_t)nranks, sizeof(slab_rank));
    const int32_t local_nrow = nx * ny * nz, total_nrow = local_nrow * nranks;
    int32_t *offsets = ialloc(nranks);
    for (int32_t q = 0; q < nranks; ++q)
        offsets[q] = local_nrow * q + 1; /* global_index_offsets (:320-324) */
    for (int32_t q = 0; q < nranks; ++q) {
        slab_rank *R = &P->r[q];
        R->local_nrow = local_nrow;
        R->start_row = local_nrow * q + 1;
        R->stop_row = R->start_row + local_nrow - 1;
        R->rowindex = ialloc(local_nrow + 1);
        R->colindex = ialloc(27 * (int64_t)local_nrow);
        R->values = (double *)calloc(27 * (size_t)local_nrow, sizeof(double));
        double *x = (double *)malloc(sizeof(double) * (size_t)local_nrow);
        double *b = (double *)malloc(sizeof(double) * (size_t)local_nrow);
        double *xe = (double *)malloc(sizeof(double) * (size_t)local_nrow);
        R->nnz = orc_generate_matrix_rank(nx, ny, nz, q, nranks, R->rowindex, R->colindex, R->values, x, b,
                                          xe);
        free(x);
        free(b);
        free(xe);
        if (mode == 0)
            local_part_mpi(R, nranks, offsets, total_nrow);
        else
            local_part_get(R, nranks, total_nrow);
    }
    if (mode == 0)
        for (int32_t q = 0; q < nranks; ++q)
            send_part_mpi(P, q);
    free(offsets);
    return P;
}

void orc_slab_plan_destroy(orc_slab_plan *P)
{
    if (!P)
        return;
    for (int32_t q = 0; q < P->nranks; ++q) {
        slab_rank *R = &P->r[q];
        free(R->rowindex), free(R->colindex), free(R->values), free(R->external_index);
        free(R->external_processor), free(R->neighbors), free(R->recv_length);
        free(R->recv_length_literal), free(R->send_length), free(R->elements_to_send);
        free(R->blk_image), free(R->blk_start), free(R->blk_inmin), free(R->blk_inmax);
        free(R->remote_index);
    }
    free(P->r);
    free(P);
}

static int32_t copy_out(int32_t *out, const int32_t *src, int32_t n)
{
    if (out)
        memcpy(out, src, sizeof(int32_t) * (size_t)(n > 0 ? n : 0));
    return n;
}

int32_t orc_slab_plan_get(const orc_slab_plan *P, int32_t rank, int32_t what, int32_t *out)
{
    const slab_rank *R = &P->r[rank];
    switch (what) {
    case ORC_SLAB_NNZ:
        return (int32_t)R->nnz;
    case ORC_SLAB_COLINDEX:
        return copy_out(out, R->colindex, (int32_t)R->nnz);
    case ORC_SLAB_ROWINDEX:
        return copy_out(out, R->rowindex, R->local_nrow + 1);
    case ORC_SLAB_EXTERNALS:
        return copy_out(out, R->external_index + 1, R->num_external);
    case ORC_SLAB_EXTERNAL_OWNERS:
        return copy_out(out, R->external_processor + 1, R->num_external);
    case ORC_SLAB_NEIGHBORS:
        return copy_out(out, R->neighbors, R->num_neighbors);
    case ORC_SLAB_RECV_LENGTH:
        return copy_out(out, R->recv_length, R->num_neighbors);
    case ORC_SLAB_RECV_LENGTH_LITERAL:
        return copy_out(out, R->recv_length_literal, R->num_neighbors);
    case ORC_SLAB_SEND_LENGTH:
        return copy_out(out, R->send_length, R->num_neighbors);
    case ORC_SLAB_ELEMENTS_TO_SEND:
        if (!R->elements_to_send)
            return 0;                   /* the CAF-V2 form sends nothing */
        return copy_out(out, R->elements_to_send + 1, R->total_to_be_sent);
    case ORC_SLAB_BLOCKS:
        if (out)
            for (int32_t k = 1; k <= R->num_blocks; ++k) {
                out[4 * (k - 1)] = R->blk_image[k];
                out[4 * (k - 1) + 1] = R->blk_start[k];
                out[4 * (k - 1) + 2] = R->blk_inmin[k];
                out[4 * (k - 1) + 3] = R->blk_inmax[k];
            }
        return R->num_blocks;
    case ORC_SLAB_REMOTE_INDEX:
        if (!R->remote_index)
            return 0;                   /* the MPI form has no block gets */
        return copy_out(out, R->remote_index + 1, R->num_external);
    default:
        return -1;
    }
}

/* exchange_externals for every rank: x[q] has local_ncol entries. */
static void exchange(const orc_slab_plan *P, double **x)
{
    for (int32_t q = 0; q < P->nranks; ++q) {
        const slab_rank *R = &P->r[q];
        if (P->mode == 0) {
            /* MPI/src/SparseMatrix.F90:647-676: the neighbour's send_buffer
             * segment for q lands at x(local_nrow+1+offset) */
            int32_t offset = 0;
            for (int32_t i = 0; i < R->num_neighbors; ++i) {
                const int32_t nb = R->neighbors[i];
                const slab_rank *N = &P->r[nb];
                int32_t soff = 0, slot = -1;
                for (int32_t k = 0; k < N->num_neighbors; ++k) {
                    if (N->neighbors[k] == q) {
                        slot = k;
                        break;
                    }
                    soff += N->send_length[k];
                }
                for (int32_t k = 0; slot >= 0 && k < N->send_length[slot]; ++k)
                    x[q][R->local_nrow + offset + k] = x[nb][N->elements_to_send[1 + soff + k] - 1];
                offset += R->recv_length[i];
            }
        } else {
            /* CAF-V2/src/SparseMatrix.F90:357-367: one contiguous range per block */
            for (int32_t k = 1; k <= R->num_blocks; ++k) {
                const double *xl = x[R->blk_image[k]] + (R->blk_inmin[k] - 1);
                for (int32_t i = R->blk_start[k]; i <= R->blk_start[k + 1] - 1; ++i)
                    x[q][R->local_nrow + i - 1] = xl[R->remote_index[i] - R->blk_inmin[k]];
            }
        }
    }
}

static double allreduce(const double *v, int32_t n)
{
    double s = v[0];
    for (int32_t q = 1; q < n; ++q)
        s = s + v[q];
    return s;
}

/* MPI/src/numerics.F90:41-162 with every rank in step: the exchange before
 * each spmv (:93-95, :129) and the dot products summed over ranks
 * (vector_operations.F90:64-65, 96-97).  b and x are the ranks' vectors one
 * after another (nranks * local_nrow); x is updated in place. */
int orc_cg_slabs(const orc_slab_plan *P, const double *b, double *x, int32_t max_iter, double tolerance,
                 int32_t *niters, double *normr_out, double *hist)
{
    const int32_t nr = P->nranks, n = P->r[0].local_nrow;
    double **p = (double **)malloc(sizeof(double *) * (size_t)nr);
    double **r = (double **)malloc(sizeof(double *) * (size_t)nr);
    double **Ap = (double **)malloc(sizeof(double *) * (size_t)nr);
    double *loc = (double *)calloc((size_t)nr, sizeof(double));
    for (int32_t q = 0; q < nr; ++q) {
        p[q] = (double *)calloc((size_t)P->r[q].local_ncol + 1, sizeof(double));
        r[q] = (double *)malloc(sizeof(double) * (size_t)n);
        Ap[q] = (double *)malloc(sizeof(double) * (size_t)n);
    }
    double normr, rtrans, oldrtrans, alpha, beta;
    int32_t it = 0;
    for (int32_t q = 0; q < nr; ++q)
        orc_vcopy(n, x + (size_t)q * n, p[q]);
    exchange(P, p);
    for (int32_t q = 0; q < nr; ++q) {
        const slab_rank *R = &P->r[q];
        orc_spmv(n, R->rowindex, R->colindex, R->values, p[q], Ap[q]);
        orc_waxpby(n, 1.0, b + (size_t)q * n, -1.0, Ap[q], r[q]);
        loc[q] = orc_ddot1(n, r[q]);
    }
    rtrans = allreduce(loc, nr);
    normr = sqrt(rtrans);
    if (hist)
        hist[0] = normr;
    for (int32_t k = 1; k <= max_iter; ++k) {
        if (normr < tolerance)
            break;
        if (k == 1) {
            for (int32_t q = 0; q < nr; ++q)
                orc_vcopy(n, r[q], p[q]);
        } else {
            oldrtrans = rtrans;
            for (int32_t q = 0; q < nr; ++q)
                loc[q] = orc_ddot1(n, r[q]);
            rtrans = allreduce(loc, nr);
            beta = rtrans / oldrtrans;
            for (int32_t q = 0; q < nr; ++q)
                orc_wxbw(n, r[q], beta, p[q]);
        }
        normr = sqrt(rtrans);
        if (hist)
            hist[k] = normr;
        exchange(P, p);
        for (int32_t q = 0; q < nr; ++q) {
            const slab_rank *R = &P->r[q];
            orc_spmv(n, R->rowindex, R->colindex, R->values, p[q], Ap[q]);
            loc[q] = orc_ddot(n, p[q], Ap[q]);
        }
        alpha = allreduce(loc, nr);
        alpha = rtrans / alpha;
        for (int32_t q = 0; q < nr; ++q) {
            orc_wwpby(n, -alpha, Ap[q], r[q]);
            orc_wwpby(n, alpha, p[q], x + (size_t)q * n);
        }
        it = k;
    }
    *niters = it;
    *normr_out = normr;
    for (int32_t q = 0; q < nr; ++q)
        free(p[q]), free(r[q]), free(Ap[q]);
    free(p), free(r), free(Ap), free(loc);
    return 0;
}
