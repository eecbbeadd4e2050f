/*
 * hpccg_gpu.h -- C-ABI of the B200 (sm_100a) HPCCG conjugate-gradient library.
 *
 * Drop-in boundary for the reference's single-rank CG path
 * (RRZE-HPC/HPCCG-F90, MPI variant; exchange_externals is a no-op on one rank,
 * MPI/src/SparseMatrix.F90:643-645).  Plain C types only: the Fortran host
 * binds these with ISO_C_BINDING interfaces, C/C++ hosts include this header,
 * Python binds them with ctypes.
 *
 * Conventions
 *  - Every call returns HPCCG_OK (0) or a positive HPCCG_ERR_* code; nothing
 *    aborts the process (the reference calls `stop`).
 *  - Matrices cross the boundary in the reference's layout: 1-based int32
 *    rowindex(nrow+1) / colindex(nnz), real(dp) values(nnz)
 *    (MPI/src/SparseMatrix.F90:44-64).
 *  - `d_` arguments are device pointers on the context's GPU; other array
 *    arguments are host pointers (pinned memory gives the fastest copies).
 *  - A context is used from one host thread at a time; calls on one context
 *    are serialised on its stream and return after the GPU work is done.
 */
#ifndef HPCCG_GPU_H
#define HPCCG_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HPCCG_OK 0
#define HPCCG_ERR_INVALID_ARG 1   /* null pointer, negative size, bad CSR */
#define HPCCG_ERR_CUDA 2          /* a CUDA runtime call failed */
#define HPCCG_ERR_OOM 3           /* device allocation failed */
#define HPCCG_ERR_BREAKDOWN 4     /* p'Ap <= 0, or a NaN/Inf scalar, in CG */
#define HPCCG_ERR_TIMEOUT 5       /* a bounded device-side wait gave up */
#define HPCCG_ERR_NOT_CONVERGED 6 /* a solve with a target stopped short of it */
#define HPCCG_ERR_UNSUPPORTED 7   /* option not available for this matrix */
#define HPCCG_ERR_NO_DEVICE 8     /* no CUDA device visible */
#define HPCCG_ERR_TOO_LARGE 9     /* input larger than a fixed capacity */

typedef struct hpccg_ctx hpccg_ctx;

/* Human-readable name of an HPCCG_* code. */
const char *hpccg_strerror(int code);

/* ---- matrix construction ------------------------------------------------ */

/* Host generator, bit-exact with MPI/src/SparseMatrix.F90:68-185
 * generate_matrix on one rank.  rowindex: nrow+1, colindex/values: capacity
 * 27*nrow (the reference allocates 27*nrow, :119-121), x/b/xexact: nrow,
 * nrow = nx*ny*nz.  *nnz receives the number of stored nonzeros. */
int hpccg_generate_matrix(int32_t nx, int32_t ny, int32_t nz, int32_t *rowindex,
                          int32_t *colindex, double *values, double *x, double *b,
                          double *xexact, int64_t *nnz);

/* Uploads a CSR matrix (reference layout) to the current CUDA device and
 * builds the device layouts the kernels use.  Replaces the matrix half of the
 * `type(SparseMatrixT)` argument of cg (MPI/src/numerics.F90:41-49). */
int hpccg_gpu_create(int32_t nrow, int64_t nnz, const int32_t *rowindex,
                     const int32_t *colindex, const double *values, hpccg_ctx **ctx);

/* Builds the generate_matrix(nx,ny,nz) matrix directly on the device (same
 * rows/cols/values as the host generator) and, if the pointers are non-null,
 * writes x (=0), b and xexact (=1) to DEVICE arrays of length nx*ny*nz. */
int hpccg_gpu_create_generated(int32_t nx, int32_t ny, int32_t nz, double *d_x, double *d_b,
                               double *d_xexact, hpccg_ctx **ctx);

/* Frees the context: its matrix copies, vectors, graphs, events and stream.
 * NULL is ignored. */
void hpccg_gpu_destroy(hpccg_ctx *ctx);

/* Basic facts about the context: rows, stored nonzeros, ELL width. */
int hpccg_gpu_info(const hpccg_ctx *ctx, int32_t *nrow, int64_t *nnz, int32_t *ell_width);

/* Copies the device CSR back in the reference's 1-based layout (for checks). */
int hpccg_gpu_download_csr(const hpccg_ctx *ctx, int32_t *rowindex, int32_t *colindex,
                           double *values);

/* SpMV kernel selection.  HPCCG_SPMV_AUTO picks the fastest bit-exact FP64
 * ELL kernel on first use (never the matrix-free stencil, which is opt-in);
 * the others force one kernel. */
#define HPCCG_SPMV_AUTO 0
#define HPCCG_SPMV_ELL 1        /* thread per row, column-major ELL (param: resident blocks/SM hint 2,3,4,8) */
#define HPCCG_SPMV_ELL2 2       /* two rows per thread, 16-byte loads (same param)  */
#define HPCCG_SPMV_CSR_VECTOR 3 /* warp-per-row CSR (lanes per row = param)    */
#define HPCCG_SPMV_STENCIL 4    /* matrix-free generate_matrix stencil (needs the geometry below) */
int hpccg_gpu_set_spmv(hpccg_ctx *ctx, int32_t kind, int32_t param);

/* Declares that the context's matrix is generate_matrix(nx,ny,nz)
 * (MPI/src/SparseMatrix.F90:68-185) and checks that on the device, entry by
 * entry: row pointers, column indices in order, and values (27.0 on the
 * diagonal, -1.0 elsewhere).  On success the matrix-free SpMV
 * HPCCG_SPMV_STENCIL may be selected: it forms every row sum from x alone, in
 * the CSR's term order, so y, fused dots and CG histories are bit-identical
 * to the ELL kernels' while A is never read.  Returns HPCCG_ERR_UNSUPPORTED
 * when the matrix differs (the geometry is then cleared) and
 * HPCCG_ERR_INVALID_ARG when nx*ny*nz is not the row count.  Contexts from
 * hpccg_gpu_create_generated are checked and have the geometry already. */
int hpccg_gpu_set_geometry(hpccg_ctx *ctx, int32_t nx, int32_t ny, int32_t nz);
int hpccg_gpu_get_spmv(const hpccg_ctx *ctx, int32_t *kind, int32_t *param);

/* ---- the CG entry point ------------------------------------------------- */

/* MPI/src/numerics.F90:41-162 cg(A, b, x, max_iter, tolerance, niters, normr)
 * on host arrays of length nrow.  x holds x0 on entry and the solution on
 * exit.  niters and normr follow the reference exactly (normr is the last
 * residual norm the loop computed, ||r_{niters-1}||; the stop test
 * `normr < tolerance` runs at the top of each iteration).  resid_hist
 * (nullable, length >= max_iter+1) receives [0] = Initial Residual and
 * [k] = the normr of iteration k, k = 1..niters.  The whole loop runs on the
 * device inside one CUDA graph with a device-side while condition. */
int hpccg_gpu_cg(hpccg_ctx *ctx, const double *b, double *x, int32_t max_iter,
                 double tolerance, int32_t *niters, double *normr, double *resid_hist);

/* Same as hpccg_gpu_cg on device arrays (b, x on the context's device). */
int hpccg_gpu_cg_device(hpccg_ctx *ctx, const double *d_b, double *d_x, int32_t max_iter,
                        double tolerance, int32_t *niters, double *normr,
                        double *resid_hist);

/* ---- mixed precision: FP64 iterative refinement around a low-precision CG ----
 *
 * No single reference routine: this replaces the whole `cg` call
 * (MPI/src/numerics.F90:41-162) when the caller wants time to a relative
 * residual instead of the reference's fixed iteration count.  The outer loop
 * is FP64 on the device: r = b - A x with the FP64 values (bit-exact
 * reference SpMV), stop when ||r||_2 <= rel_tol ||b||_2 (the FP64 true
 * residual alone decides convergence), else solve A d = r/||r|| with an
 * inner CG in FP32 vectors and FP32 (HPCCG_PREC_FP32) or BF16
 * (HPCCG_PREC_BF16) copies of A's values, row sums accumulated in FP32, and
 * update x += ||r|| d in FP64.  The inner CG stops at ||r_in|| <= inner_rtol
 * ||r_in,0||, or, with inner_rtol = 0, at the adaptive target
 * max(1e-5, 0.5 rel_tol ||b|| / ||r||).  Needs an ELL width <= 27.
 * Returns HPCCG_OK when the FP64 target is met, HPCCG_ERR_NOT_CONVERGED when
 * max_outer cycles did not reach it (x holds the last iterate). */
#define HPCCG_PREC_FP64 0
#define HPCCG_PREC_FP32 1
#define HPCCG_PREC_BF16 2

typedef struct hpccg_mixed_info {
  int32_t outer_iters; /* FP64 refinement cycles run                 */
  int32_t inner_iters; /* low-precision CG iterations, all cycles    */
  double relres;       /* final FP64 ||b - A x|| / ||b||             */
  int32_t status;      /* device status word (HPCCG_OK or BREAKDOWN) */
  int32_t reserved;
} hpccg_mixed_info;

int hpccg_gpu_solve_mixed(hpccg_ctx *ctx, const double *b, double *x, int32_t precision,
                          double rel_tol, int32_t max_outer, int32_t max_inner, double inner_rtol,
                          hpccg_mixed_info *info);
int hpccg_gpu_solve_mixed_device(hpccg_ctx *ctx, const double *d_b, double *d_x, int32_t precision,
                                 double rel_tol, int32_t max_outer, int32_t max_inner,
                                 double inner_rtol, hpccg_mixed_info *info);

/* y = A x with the low-precision values (FP32 vectors), for checks/timing. */
int hpccg_gpu_spmv_lowp(hpccg_ctx *ctx, int32_t precision, const float *d_x, float *d_y);

/* Rows per thread (1, 2 or 4) of the low-precision SpMV for one precision. */
int hpccg_gpu_set_mixed_rows_per_thread(hpccg_ctx *ctx, int32_t precision, int32_t rpt);

/* Average ms of the inner-CG kernels (p update, low-precision SpMV + p.Ap,
 * r update + r.r), each launched `reps` times back to back.  When the inner
 * iteration is one fused pass (hpccg_gpu_mixed_fused), ms[1] is that pass,
 * ms[0] the FP64 refinement residual of an outer cycle and ms[2] = 0. */
int hpccg_gpu_time_mixed_kernels(hpccg_ctx *ctx, int32_t precision, int32_t reps, float *ms);

/* The fused inner iteration of the matrix-free solve (HPCCG_SPMV_STENCIL
 * contexts with nx % 4 == 0): one TMA-fed pass per CG iteration reads r, p
 * and d and writes r, p and d (24 bytes per row instead of 40).  A p of the
 * previous iteration is recomputed from p with a two-deep halo instead of
 * being stored, and the next beta comes from the recurrence
 * ||r - alpha Ap||^2 = r.r - 2 alpha r.Ap + alpha^2 Ap.Ap.  On by default;
 * set_mixed_fused(ctx, 0) selects the three-kernel iteration.  mixed_fused
 * reports whether the inner solves of ctx use it. */
int hpccg_gpu_set_mixed_fused(hpccg_ctx *ctx, int32_t on);
int hpccg_gpu_mixed_fused(hpccg_ctx *ctx, int32_t *fused);

/* One fused pass on caller buffers (FP32, device, nrow each), for checks:
 * with Ap = A p, r' = first ? r : r - alpha Ap, p' = first ? r : r' + beta p,
 * d += alpha p (d = 0 when first), Ap' = A p'; writes r', p', d and returns
 * dots = {p'.Ap', r'.Ap', Ap'.Ap', r'.r'}.  HPCCG_ERR_UNSUPPORTED when the
 * context has no fused iteration. */
int hpccg_gpu_mixed_pass(hpccg_ctx *ctx, const float *d_r, const float *d_p, float *d_d, float *d_r_out,
                         float *d_p_out, double alpha, double beta, int32_t first, double dots[4]);

/* ---- batched solves of many independent systems ------------------------
 *
 * No single reference routine: the reference solves one system per run.  A
 * batch stacks independent systems block-diagonally (each system's rows start
 * on a 512-row boundary of one "stacked" vector).  One persistent kernel per
 * CG phase walks tiles of every system that is still active; the loop runs
 * on the device in one CUDA graph.  Each system stops on its own at
 * ||b_s - A_s x_s|| <= rel_tol ||b_s||.  Dot products are reduced per
 * 512-row chunk in a fixed order, so results do not depend on the tile
 * schedule the autotuner picks. */
typedef struct hpccg_batch hpccg_batch;

/* generate_matrix systems: sizes[3s..3s+2] = nx, ny, nz of system s. */
int hpccg_batch_create_generated(int32_t nsys, const int32_t *sizes, hpccg_batch **batch);
/* Systems given as reference-layout CSRs (1-based; at most 27 entries a row). */
int hpccg_batch_create(int32_t nsys, const int32_t *nrows, const int32_t *const *rowindex,
                       const int32_t *const *colindex, const double *const *values,
                       hpccg_batch **batch);
void hpccg_batch_destroy(hpccg_batch *batch);
/* stacked_rows: length of the stacked vectors; row_offsets (nullable, 2*nsys):
 * [2s] = first stacked row of system s, [2s+1] = its row count. */
int hpccg_batch_info(const hpccg_batch *batch, int32_t *nsys, int64_t *stacked_rows,
                     int64_t *row_offsets);
/* Tile size in 512-row chunks and resident blocks per SM of the phase
 * kernels; (0, 0) re-enables the autotuner (run on the next solve). */
int hpccg_batch_set_schedule(hpccg_batch *batch, int32_t tile_chunks, int32_t blocks_per_sm);
/* Row kernel of the batch: HPCCG_SPMV_ELL (default; the stacked matrix) or
 * HPCCG_SPMV_STENCIL (matrix-free rows from each system's grid, reference term
 * order, so FP64 iterates are bit-identical; only for batches from
 * hpccg_batch_create_generated, else HPCCG_ERR_UNSUPPORTED).  A change of kind
 * re-runs the schedule autotuner on the next solve. */
int hpccg_batch_set_spmv(hpccg_batch *batch, int32_t kind);
int hpccg_batch_get_schedule(const hpccg_batch *batch, int32_t *tile_chunks, int32_t *blocks_per_sm);
/* y = A x over all systems (stacked device vectors). */
int hpccg_batch_spmv(hpccg_batch *batch, const double *d_x, double *d_y);
/* Solves every system.  d_b / d_x are stacked device vectors (x: x0 in,
 * solution out).  precision HPCCG_PREC_FP64: CG per system (max_iter caps the
 * iterations); HPCCG_PREC_FP32 / HPCCG_PREC_BF16: per-system FP64 iterative
 * refinement around an inner CG (max_iter caps each inner solve, at most 30
 * cycles).  Host outputs (nullable, nsys each): iterations (inner iterations
 * for the refinement solvers), final FP64 relative residual, refinement
 * cycles.  Returns HPCCG_ERR_NOT_CONVERGED if any system missed rel_tol. */
int hpccg_batch_solve(hpccg_batch *batch, const double *d_b, double *d_x, int32_t precision,
                      double rel_tol, int32_t max_iter, int32_t *iters, double *relres,
                      int32_t *outer);
/* The same with HOST arrays b and x (stacked layout, length stacked_rows):
 * the library copies them in and the solution out.  The call a host driver
 * makes, like hpccg_gpu_cg for one system. */
int hpccg_batch_solve_host(hpccg_batch *batch, const double *b, double *x, int32_t precision,
                           double rel_tol, int32_t max_iter, int32_t *iters, double *relres,
                           int32_t *outer);
/* Device ms of the last hpccg_batch_solve (events around the graph launch). */
int hpccg_batch_last_solve_ms(const hpccg_batch *batch, float *ms);

/* ---- learned preconditioner: a 3D U-Net -----------------------------------
 *
 * No reference counterpart (the reference's CG is unpreconditioned).  A
 * 4-level U-Net with 16 channels at every level (104,337 parameters), BF16
 * activations on tcgen05 tensor cores with FP32 accumulation, FP32 master
 * weights; input and output are one FP32 channel on an nx*ny*nz grid (each a
 * multiple of 8), batches stacked along a slowest batch dimension. */
typedef struct hpccg_unet hpccg_unet;

/* He-uniform weights from the project's generator (seed), zero biases. */
int hpccg_unet_create(uint64_t seed, hpccg_unet **unet);
void hpccg_unet_destroy(hpccg_unet *unet);
int hpccg_unet_num_params(const hpccg_unet *unet, int64_t *nparams);
/* Flat FP32 parameter vector (host), layer by layer: W[27][cin][16], bias[16];
 * then the 16->1 projection (16 weights, 1 bias). */
int hpccg_unet_get_params(const hpccg_unet *unet, float *host_params);
int hpccg_unet_set_params(hpccg_unet *unet, const float *host_params);
/* out = net(in) for nb stacked grids (device FP32 arrays of nb*nx*ny*nz). */
int hpccg_unet_forward(hpccg_unet *unet, int32_t nx, int32_t ny, int32_t nz, int32_t nb, const float *d_in,
                       float *d_out);
/* Mean squared error against d_target and its gradient w.r.t. every
 * parameter (kept on the device; copied to grad_host when non-null). */
int hpccg_unet_loss_grad(hpccg_unet *unet, int32_t nx, int32_t ny, int32_t nz, int32_t nb, const float *d_in,
                         const float *d_target, float *loss, float *grad_host);
/* Loss of hpccg_unet_loss_grad: 0 = mean squared error (default), 1 = energy
 * norm (1/n) d.(A d), d = target - out, with A the generate_matrix operator
 * on the same grid -- the norm in which CG measures the error. */
int hpccg_unet_set_loss(hpccg_unet *unet, int32_t kind);
/* One Adam update with the gradient of the last hpccg_unet_loss_grad. */
int hpccg_unet_adam_step(hpccg_unet *unet, float lr, float beta1, float beta2, float eps);
/* Average ms of `reps` forward passes on one grid. */
int hpccg_unet_time_forward(hpccg_unet *unet, int32_t nx, int32_t ny, int32_t nz, int32_t reps,
                            const float *d_in, float *d_out, float *ms);
/* One 3x3x3 conv layer with 16 outputs, for tests: BF16 inputs in the
 * row-planar layout [b][z][y][half][x][8 channels] (nin = 1 or 2 groups of 16
 * channels; 16-channel outputs use the same layout), weights FP32 [27][16*nin][16],
 * epi 0 = bias+ReLU (BF16 out), 1 = bias (BF16), 2 = bias+ReLU then the 16->1
 * projection d_proj (FP32 out), 3 = raw FP32 16-channel out; path 0 =
 * tcgen05 (row tiles when nx is a multiple of 128), 1 = CUDA cores,
 * 2 = tcgen05 with brick tiles (per-tap fetches).  nin = 0 is the network's
 * 1-channel input layer: d_in0 an FP32 grid [b][z][y][x], weights FP32 [27][16],
 * epi 0 or 1; path 0 = tcgen05 (nx a multiple of 128, else
 * HPCCG_ERR_UNSUPPORTED), 1 = CUDA cores. */
int hpccg_unet_conv3_layer(int32_t nx, int32_t ny, int32_t nz, int32_t nb, int32_t nin, const void *d_in0,
                           const void *d_in1, const float *d_w, const float *d_bias, const float *d_proj,
                           int32_t epi, int32_t path, void *d_out);

/* Flexible (Polak-Ribiere) preconditioned CG on the nx*ny*nz grid of the
 * context's generate_matrix system, preconditioner z = s * net(r/s) with
 * s = rms(r).  All vectors, dot products and the convergence test are FP64;
 * plain CG (z = r) takes over when the preconditioned iteration stalls (no
 * 10% residual reduction in 5 iterations) or r.z <= 0, and the FP64 true
 * residual b - A x decides convergence.  unet = NULL runs plain CG.  Device
 * arrays; x holds x0 on entry. */
typedef struct hpccg_fcg_info {
  int32_t iters;      /* CG iterations (SpMVs) */
  int32_t nn_applies; /* network applications */
  int32_t fallback;   /* 1 if plain CG took over */
  int32_t status;
  double relres;      /* final FP64 ||b - A x|| / ||b|| */
} hpccg_fcg_info;
int hpccg_gpu_solve_fcg(hpccg_ctx *ctx, hpccg_unet *unet, int32_t nx, int32_t ny, int32_t nz, const double *d_b,
                        double *d_x, double rel_tol, int32_t max_iter, hpccg_fcg_info *info);

/* The learned preconditioner inside mixed precision: FP64 iterative
 * refinement (r = b - A x with the context's FP64 SpMV, stop at
 * ||r|| <= rel_tol ||b||, x += ||r|| d) around a flexible (Polak-Ribiere) CG
 * with FP32 vectors, the FP32 matrix-free operator and z = s * net(r/s); the
 * inner solve stops at max(1e-5, 0.5 rel_tol ||b|| / ||r||) relative, plain
 * CG takes over as in hpccg_gpu_solve_fcg, unet = NULL runs plain FP32 CG.
 * Needs the context's geometry (hpccg_gpu_set_geometry or a generated
 * context) equal to nx, ny, nz (multiples of 8 with a network), else
 * HPCCG_ERR_UNSUPPORTED.  Device arrays; x holds x0 on entry.  No reference
 * counterpart: it replaces the whole cg call (MPI/src/numerics.F90:41-162)
 * with a time-to-tolerance solve. */
typedef struct hpccg_mixed_fcg_info {
  int32_t outer_iters; /* FP64 refinement cycles          */
  int32_t inner_iters; /* FP32 flexible-CG iterations     */
  int32_t nn_applies;  /* network applications            */
  int32_t fallback;    /* 1 if plain CG took over         */
  int32_t status;
  int32_t reserved;
  double relres;       /* final FP64 ||b - A x|| / ||b||  */
} hpccg_mixed_fcg_info;
int hpccg_gpu_solve_mixed_fcg(hpccg_ctx *ctx, hpccg_unet *unet, int32_t nx, int32_t ny, int32_t nz,
                              const double *d_b, double *d_x, double rel_tol, int32_t max_outer, int32_t max_inner,
                              hpccg_mixed_fcg_info *info);

/* ---- op-level drop-ins (device arrays), MPI/src/SparseMatrix.F90:213-232
 *      and MPI/src/vector_operations.F90:40-169 ------------------------------ */

int hpccg_gpu_spmv(hpccg_ctx *ctx, const double *d_x, double *d_y);      /* y = A x   */
int hpccg_gpu_ddot(hpccg_ctx *ctx, int32_t n, const double *d_x, const double *d_y,
                   double *result);                                          /* x.y       */
int hpccg_gpu_ddot1(hpccg_ctx *ctx, int32_t n, const double *d_x, double *result); /* x.x */
int hpccg_gpu_waxpby(hpccg_ctx *ctx, int32_t n, double alpha, const double *d_x, double beta,
                     const double *d_y, double *d_w);                       /* w=ax+by   */
int hpccg_gpu_wwpby(hpccg_ctx *ctx, int32_t n, double beta, const double *d_y,
                    double *d_w);                                            /* w=w+by    */
int hpccg_gpu_wxbw(hpccg_ctx *ctx, int32_t n, const double *d_x, double beta,
                   double *d_w);                                             /* w=x+bw    */
int hpccg_gpu_vcopy(hpccg_ctx *ctx, int32_t n, const double *d_x, double *d_y); /* y = x */

/* ---- synthetic inputs -------------------------------------------------- */

/* d_out[i] = uniform double in [-1,1) from the project's counter-based
 * generator: z = splitmix64 finaliser of seed + (offset+i+1)*0x9E3779B97F4A7C15,
 * value = 2*((z>>11)*2^-53) - 1.  No reference counterpart (the reference
 * only uses x = 1); it makes the random right-hand sides reproducible on
 * host and device. */
int hpccg_gpu_uniform_pm1(hpccg_ctx *ctx, uint64_t seed, int64_t offset, int64_t n, double *d_out);

/* ---- several ranks: z slabs of the weak-scaled problem -------------------
 *
 * With nranks ranks the reference gives rank r the rows
 * local_nrow*r+1 .. local_nrow*(r+1) of the nx x ny x (nz*nranks) grid
 * (MPI/src/SparseMatrix.F90:68-185, start_row at :112), renumbers each rank's
 * columns into its own rows followed by externals owned by other ranks
 * (make_local_matrix, :235-627), fills p's externals before every SpMV
 * (exchange_externals, :630-680) and sums each dot product over the ranks
 * (MPI/src/vector_operations.F90:64-65, 96-97).  Two halo forms:
 * HPCCG_HALO_MPI, externals grouped by owner and a send list per neighbour
 * (the MPI variant); HPCCG_HALO_GET, externals in order of first appearance,
 * each run of one owner filled from one contiguous range of the owner's
 * vector (CAF-V2/src/SparseMatrix.F90:205-370).  Block lengths are the block
 * sizes; the MPI variant's counting loop (:533-545) gives one more for every
 * block but a rank's last, so with three or more ranks its middle ranks
 * would read shifted halos. */
#define HPCCG_HALO_MPI 0
#define HPCCG_HALO_GET 1

/* generate_matrix on rank `rank` of `nranks` (global 1-based columns, z
 * truncated only at the global ends); hpccg_generate_matrix is rank 0 of 1. */
int hpccg_generate_matrix_rank(int32_t nx, int32_t ny, int32_t nz, int32_t rank, int32_t nranks,
                               int32_t *rowindex, int32_t *colindex, double *values, double *x, double *b,
                               double *xexact, int64_t *nnz);

/* The halo plan of one rank (host memory only; no GPU needed).  rowindex /
 * colindex: the rank's rows in the reference layout with GLOBAL 1-based
 * columns; first_rows[q] = first global row of rank q (1-based), q = 0..nranks,
 * first_rows[nranks] = total rows + 1 (the reference's global_index_offsets,
 * :318-324).  HPCCG_HALO_MPI plans need the neighbours' requests
 * (hpccg_slab_plan_set_sends) before hpccg_slab_create; HPCCG_HALO_GET plans
 * are complete at once. */
typedef struct hpccg_slab_plan hpccg_slab_plan;
int hpccg_slab_plan_create(int32_t nrow, int64_t nnz, const int32_t *rowindex, const int32_t *colindex,
                           int32_t nranks, int32_t rank, const int32_t *first_rows, int32_t halo_mode,
                           hpccg_slab_plan **plan);
void hpccg_slab_plan_destroy(hpccg_slab_plan *plan);
/* total_to_send is -1 until the sends are set (HPCCG_HALO_MPI). */
int hpccg_slab_plan_info(const hpccg_slab_plan *plan, int32_t *num_external, int32_t *num_neighbors,
                         int32_t *num_blocks, int32_t *total_to_send);
/* HPCCG_HALO_MPI: neighbours in receive order and the externals each sends. */
int hpccg_slab_plan_neighbors(const hpccg_slab_plan *plan, int32_t *neighbors, int32_t *recv_length);
/* Global id and owning rank of each local external, in local order (for
 * HPCCG_HALO_MPI the ids to send to each neighbour, block by block:
 * make_local_matrix's new_external, :512-514). */
int hpccg_slab_plan_externals(const hpccg_slab_plan *plan, int32_t *global_ids, int32_t *owners);
/* HPCCG_HALO_MPI: what each neighbour (in this rank's neighbour order) asked
 * for, as global ids, concatenated; stored as elements_to_send (local,
 * :605-607).  Ids outside this rank's rows are rejected. */
int hpccg_slab_plan_set_sends(hpccg_slab_plan *plan, const int32_t *send_length, const int32_t *global_ids);
int hpccg_slab_plan_sends(const hpccg_slab_plan *plan, int32_t *send_length, int32_t *elements_to_send);
/* The rank's columns renumbered: 1..nrow own rows, nrow+1.. externals. */
int hpccg_slab_plan_colindex(const hpccg_slab_plan *plan, int32_t *colindex_local);
/* HPCCG_HALO_GET: 4 per block (owner rank, first external (1-based), inmin,
 * inmax in the owner's local rows) and each external's owner-local row. */
int hpccg_slab_plan_blocks(const hpccg_slab_plan *plan, int32_t *blocks, int32_t *remote_index);

/* The rank's device part on the current GPU: the local matrix (values in the
 * CSR order of the plan's rowindex) as a column-major ELL over
 * [own rows | externals], the send list or the block lists.  Vectors that
 * SpMV reads (p) hold ncol = nrow + externals entries. */
typedef struct hpccg_slab hpccg_slab;
int hpccg_slab_create(const hpccg_slab_plan *plan, const double *values, hpccg_slab **slab);
void hpccg_slab_destroy(hpccg_slab *slab);
int hpccg_slab_info(const hpccg_slab *slab, int32_t *nrow, int32_t *ncol, int32_t *total_to_send,
                    int32_t *num_blocks);
/* y = A x (x: ncol entries), the reference's term order. */
int hpccg_slab_spmv(hpccg_slab *slab, const double *d_x, double *d_y);
/* HPCCG_HALO_MPI exchange: d_sendbuf[i] = x(elements_to_send(i)), neighbour
 * after neighbour (:664-666); the receiver puts neighbour i's part at
 * x + nrow + (recv_length of the neighbours before i). */
int hpccg_slab_pack(hpccg_slab *slab, const double *d_x, double *d_sendbuf);
/* HPCCG_HALO_GET exchange: d_range holds the owner's rows inmin..inmax of
 * `block`; scatters them into the block's externals of x (:360-367). */
int hpccg_slab_scatter_block(hpccg_slab *slab, int32_t block, const double *d_range, double *d_x);

/* One rank's CG (MPI/src/numerics.F90:41-162) as steps between which the
 * caller moves data: after START and BEGIN it fills p's externals, after
 * PREPARE, SPMV and UPDATE it sets d_state[1] to the sum over ranks of every
 * rank's d_state[0] (in rank order).  d_state: 8 doubles on the device,
 * [0] local dot, [1] its sum over ranks, [2] rtrans, [3] normr, [4] alpha,
 * [5] beta, [6] done (set by BEGIN once normr < tolerance; later steps do
 * nothing), [7] tolerance (set by the caller).  Vectors: b, x, r, Ap nrow
 * entries, p ncol.  d_hist (nullable): [0] and [k] as in hpccg_gpu_cg.
 * Sequence: START; exchange p; PREPARE; sum; PREPARED; then for k = 1, 2, ..:
 * BEGIN(k); exchange p; SPMV; sum; UPDATE; sum -- until done. */
#define HPCCG_SLAB_START 0    /* p = x */
#define HPCCG_SLAB_PREPARE 1  /* Ap = A p, r = b - Ap, [0] = local r.r */
#define HPCCG_SLAB_PREPARED 2 /* rtrans = [1], normr = sqrt(rtrans) */
#define HPCCG_SLAB_BEGIN 3    /* stop test; p = r (k = 1) or beta = [1]/rtrans, p = r + beta p */
#define HPCCG_SLAB_SPMV 4     /* Ap = A p, [0] = local p.Ap */
#define HPCCG_SLAB_UPDATE 5   /* alpha = rtrans/[1]; r -= alpha Ap; x += alpha p; [0] = local r.r */
int hpccg_slab_cg_step(hpccg_slab *slab, int32_t step, int32_t k, const double *d_b, double *d_x, double *d_p,
                       double *d_r, double *d_Ap, double *d_state, double *d_hist);

/* All nslabs ranks in this process (slabs[q] is rank q, each on its own GPU
 * or several on one): the whole CG with the exchange done by device copies
 * and the sums folded in rank order.  d_b[q], d_x[q]: rank q's vectors on its
 * GPU.  niters, normr and resid_hist as in hpccg_gpu_cg. */
int hpccg_slab_group_cg(hpccg_slab *const *slabs, int32_t nslabs, const double *const *d_b, double *const *d_x,
                        int32_t max_iter, double tolerance, int32_t *niters, double *normr, double *resid_hist);
/* The same with HOST arrays: b[q] and x[q] (in: x0, out: x) hold rank q's
 * nrow rows.  The library copies them to each rank's GPU and back, as
 * hpccg_gpu_cg does for one rank; the call a host driver of all the ranks makes. */
int hpccg_slab_group_cg_host(hpccg_slab *const *slabs, int32_t nslabs, const double *const *b, double *const *x,
                             int32_t max_iter, double tolerance, int32_t *niters, double *normr,
                             double *resid_hist);

/* ---- allocation-free entry point ---------------------------------------- */

/* Dot product x.y of two device arrays that allocates no device memory.  This
 * entry point has no counterpart in the reference.  It exists for callers that
 * cannot let a library call cudaMalloc: hosts whose own memory manager owns
 * all device memory (a pre-sized pool or a caching allocator the whole
 * process must use), and code that may not allocate after its set-up phase
 * (cudaMalloc can synchronise the device and can fail on a fragmented heap).
 * It needs no hpccg_ctx.  The partial sums live in a fixed 512 KiB array
 * compiled into the library, which every GPU that loads the library keeps
 * until the process exits; so n is limited to 134,217,728 elements and larger
 * n returns HPCCG_ERR_TOO_LARGE.  The work runs on `stream` (a cudaStream_t;
 * NULL = the legacy default stream) on the current device, and the call
 * returns after *result (host memory) is written.  Every call looks up the
 * array's device address on the current device (cudaGetSymbolAddress); the
 * first call on a device also loads the library's kernels there, so make that
 * first call before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (from several host threads or
 * streams at once) race and must be serialised by the caller. */
int hpccg_gpu_ddot_noalloc(int32_t n, const double *d_x, const double *d_y, double *result,
                           void *stream);

/* ---- timing helpers (device time, CUDA events on the context stream) ----- */

/* Device time in ms of the last hpccg_gpu_cg / hpccg_gpu_cg_device solve,
 * from events recorded on the context stream around the graph launch (input
 * and output copies excluded). */
int hpccg_gpu_last_solve_ms(const hpccg_ctx *ctx, float *ms);

/* Average device time in ms of each CG iteration kernel launched `reps` times
 * back to back on the context stream: ms[0] = p/x update, ms[1] = SpMV fused
 * with p.Ap, ms[2] = r update fused with r.r.  Leaves the CG work vectors
 * with unspecified contents. */
int hpccg_gpu_time_cg_kernels(hpccg_ctx *ctx, int32_t reps, float *ms);

/* Average device time in ms of `reps` back-to-back SpMVs y = A x with the
 * current kernel selection. */
int hpccg_gpu_time_spmv(hpccg_ctx *ctx, const double *d_x, double *d_y, int32_t reps,
                        float *ms_per_call);

#ifdef __cplusplus
}
#endif
#endif /* HPCCG_GPU_H */
