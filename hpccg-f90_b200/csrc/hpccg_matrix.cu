// hpccg_matrix.cu -- matrix construction, upload, device layouts, context life cycle.
//
// Reference counterparts: generate_matrix (MPI/src/SparseMatrix.F90:68-185) and
// the SparseMatrixT container (:44-64).  One rank: start_row = 1, total_nrow =
// nx*ny*nz, so the z bound curcol in [1,total_nrow] clips the first/last z plane.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "hpccg_rows.cuh"

namespace hpccg {

static thread_local char g_last_error[512];

int set_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  snprintf(g_last_error, sizeof(g_last_error), "%s failed at %s:%d: %s", what, file, line,
           cudaGetErrorString(e));
  if (getenv("HPCCG_VERBOSE")) fprintf(stderr, "hpccg: %s\n", g_last_error);
  return e == cudaErrorMemoryAllocation ? HPCCG_ERR_OOM : HPCCG_ERR_CUDA;
}

// Number of stencil neighbours kept along one axis for 1-based position i of n.
__host__ __device__ inline int axis_count(int i, int n) { return 1 + (i > 1) + (i < n); }
// Entries contributed by positions 1..i-1 along one axis.
__host__ __device__ inline int64_t axis_prefix(int i, int n) {
  int64_t s = 0;
  if (i > 1) s = (n >= 2) ? (int64_t)(3 * i - 4) : 0;  // 2 + 3*(i-2): first slot has 2
  return s;
}
__host__ __device__ inline int64_t axis_total(int n) { return n >= 2 ? 3 * (int64_t)n - 2 : 1; }

// Row start (0-based) of 1-based grid point (ix,iy,iz) in generate_matrix's
// CSR: rows run iz -> iy -> ix and the kept-neighbour count is separable.
__host__ __device__ inline int64_t row_start(int ix, int iy, int iz, int nx, int ny, int nz) {
  const int64_t tx = axis_total(nx), ty = axis_total(ny);
  const int cz = axis_count(iz, nz), cy = axis_count(iy, ny);
  return axis_prefix(iz, nz) * ty * tx + (int64_t)cz * (axis_prefix(iy, ny) * tx +
                                                      (int64_t)cy * axis_prefix(ix, nx));
}

// Writes row `row` (0-based) of generate_matrix into CSR and ELL layouts.
// Neighbour order sz -> sy -> sx ascending, as MPI/src/SparseMatrix.F90:146-148.
__global__ void generate_kernel(int nx, int ny, int nz, int32_t *rowptr, int32_t *col,
                                double *val, int32_t *ell_col, double *ell_val, int npad,
                                int W, double *x, double *b, double *xexact) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(row % nx) + 1;
    const int iy = (int)((row / nx) % ny) + 1;
    const int iz = (int)(row / ((int64_t)nx * ny)) + 1;
    int64_t cur = row_start(ix, iy, iz, nx, ny, nz);
    rowptr[row] = (int32_t)cur;
    if (row == n - 1) rowptr[n] = (int32_t)(axis_total(nx) * axis_total(ny) * axis_total(nz));
    int k = 0;
    for (int sz = (iz > 1 ? -1 : 0); sz <= (iz < nz ? 1 : 0); ++sz)
      for (int sy = (iy > 1 ? -1 : 0); sy <= (iy < ny ? 1 : 0); ++sy)
        for (int sx = (ix > 1 ? -1 : 0); sx <= (ix < nx ? 1 : 0); ++sx) {
          const int32_t c = (int32_t)(row + (int64_t)sz * nx * ny + (int64_t)sy * nx + sx);
          const double v = (sz == 0 && sy == 0 && sx == 0) ? 27.0 : -1.0;
          col[cur] = c;
          val[cur] = v;
          ell_col[(int64_t)k * npad + row] = c;
          ell_val[(int64_t)k * npad + row] = v;
          ++cur;
          ++k;
        }
    const int nnzrow = k;
    for (; k < W; ++k) {
      ell_col[(int64_t)k * npad + row] = (int32_t)row;
      ell_val[(int64_t)k * npad + row] = 0.0;
    }
    if (x) x[row] = 0.0;
    if (b) b[row] = 27.0 - (double)(nnzrow - 1);
    if (xexact) xexact[row] = 1.0;
  }
}

// 1-based reference CSR -> 0-based device CSR, plus validation flags.
__global__ void rebase_kernel(int32_t n, int64_t nnz, int32_t *rowptr, int32_t *col,
                              int *bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += stride) {
    const int32_t v = rowptr[i] - 1;
    rowptr[i] = v;
  }
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += stride) {
    const int32_t c = col[j];
    if (c < 1 || c > n) atomicOr(bad, 2);
    col[j] = c - 1;
  }
}

__global__ void check_rows_kernel(int32_t n, int64_t nnz, const int32_t *rowptr, int W,
                                  int *bad, int *maxlen) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = rowptr[i], e = rowptr[i + 1];
    if (e < a || a < 0 || e > nnz) atomicOr(bad, 1);
    else atomicMax(maxlen, e - a);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (rowptr[0] != 0 || rowptr[n] != nnz)) atomicOr(bad, 4);
}

__global__ void csr_to_ell_kernel(int32_t n, const int32_t *rowptr, const int32_t *col,
                                  const double *val, int32_t *ell_col, double *ell_val,
                                  int npad, int W) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = rowptr[i], len = rowptr[i + 1] - a;
    for (int k = 0; k < W; ++k) {
      const bool real = k < len;
      ell_col[(int64_t)k * npad + i] = real ? col[a + k] : (int32_t)i;
      ell_val[(int64_t)k * npad + i] = real ? val[a + k] : 0.0;
    }
  }
  // padding rows beyond n: point at row 0 with value 0 (never stored to y)
  for (int64_t i = n + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < W; ++k) {
      ell_col[(int64_t)k * npad + i] = 0;
      ell_val[(int64_t)k * npad + i] = 0.0;
    }
}

__global__ void pad_rows_kernel(int32_t n, int npad, int W, int32_t *ell_col, double *ell_val) {
  for (int64_t i = n + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad;
       i += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < W; ++k) {
      ell_col[(int64_t)k * npad + i] = 0;
      ell_val[(int64_t)k * npad + i] = 0.0;
    }
}

static int init_ctx_common(hpccg_ctx *c) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HPCCG_ERR_NO_DEVICE;
  HPCCG_CUDA(cudaGetDevice(&c->device));
  HPCCG_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
  HPCCG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  HPCCG_CUDA(cudaEventCreate(&c->ev0));
  HPCCG_CUDA(cudaEventCreate(&c->ev1));
  HPCCG_CUDA(cudaEventCreate(&c->solve0));
  HPCCG_CUDA(cudaEventCreate(&c->solve1));
  // Streaming kernels: a fixed grid of (resident blocks per SM) x SMs, so the
  // reduction partition -- and with it every dot product -- is reproducible.
  c->grid = std::min(kMaxPartials, c->num_sms * 8);
  HPCCG_CUDA(cudaMalloc(&c->d_partials, sizeof(double) * kMaxPartials));
  HPCCG_CUDA(cudaMalloc(&c->d_counter, sizeof(unsigned) * 16));
  HPCCG_CUDA(cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned) * 16, c->stream));
  HPCCG_CUDA(cudaMalloc(&c->d_state, sizeof(CgState)));
  return HPCCG_OK;
}

static int alloc_matrix(hpccg_ctx *c, int32_t n, int64_t nnz, int W) {
  c->nrow = n;
  c->nnz = nnz;
  c->ell_width = W;
  c->npad = (int32_t)(((int64_t)n + kEllAlign - 1) / kEllAlign * kEllAlign);
  HPCCG_CUDA(cudaMalloc(&c->d_rowptr, sizeof(int32_t) * ((size_t)n + 1)));
  HPCCG_CUDA(cudaMalloc(&c->d_col, sizeof(int32_t) * std::max<int64_t>(nnz, 1)));
  HPCCG_CUDA(cudaMalloc(&c->d_val, sizeof(double) * std::max<int64_t>(nnz, 1)));
  const size_t vec = sizeof(double) * (size_t)c->npad;
  HPCCG_CUDA(cudaMalloc(&c->d_r, vec));
  HPCCG_CUDA(cudaMalloc(&c->d_p, vec));
  HPCCG_CUDA(cudaMalloc(&c->d_Ap, vec));
  HPCCG_CUDA(cudaMalloc(&c->d_x, vec));
  HPCCG_CUDA(cudaMalloc(&c->d_b, vec));
  HPCCG_CUDA(cudaMemsetAsync(c->d_p, 0, vec, c->stream));
  return HPCCG_OK;
}

static int alloc_ell(hpccg_ctx *c) {
  if (c->ell_width <= 0 || c->ell_width > 32) return HPCCG_OK;  // CSR kernels only
  const size_t slots = (size_t)c->ell_width * (size_t)c->npad;
  HPCCG_CUDA(cudaMalloc(&c->d_ell_col, sizeof(int32_t) * slots));
  HPCCG_CUDA(cudaMalloc(&c->d_ell_val, sizeof(double) * slots));
  return HPCCG_OK;
}

int ensure_workspace(hpccg_ctx *c, int32_t hist_cap) {
  if (hist_cap > c->hist_cap) {
    if (c->d_hist) cudaFree(c->d_hist);
    c->d_hist = nullptr;
    HPCCG_CUDA(cudaMalloc(&c->d_hist, sizeof(double) * (size_t)hist_cap));
    c->hist_cap = hist_cap;
  }
  return HPCCG_OK;
}

static int grid_for(const hpccg_ctx *c, int64_t n) {
  const int64_t need = (n + kBlock - 1) / kBlock;
  return (int)std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)c->num_sms * 16));
}

}  // namespace hpccg

using namespace hpccg;

extern "C" const char *hpccg_strerror(int code) {
  switch (code) {
    case HPCCG_OK: return "ok";
    case HPCCG_ERR_INVALID_ARG: return "invalid argument";
    case HPCCG_ERR_CUDA: return g_last_error[0] ? g_last_error : "CUDA error";
    case HPCCG_ERR_OOM: return "device out of memory";
    case HPCCG_ERR_BREAKDOWN: return "CG breakdown (p'Ap <= 0 or non-finite scalar)";
    case HPCCG_ERR_TIMEOUT: return "bounded device wait timed out";
    case HPCCG_ERR_NOT_CONVERGED: return "not converged";
    case HPCCG_ERR_UNSUPPORTED: return "unsupported option";
    case HPCCG_ERR_NO_DEVICE: return "no CUDA device";
    case HPCCG_ERR_TOO_LARGE: return "input larger than the fixed capacity of this entry point";
    default: return "unknown error";
  }
}

// Host generator, same rows/cols/values/b as MPI/src/SparseMatrix.F90:68-185.
// Written per row from the kept stencil ranges of each axis; the ranges are
// visited low -> high in z, y, x so the column order equals the reference's.
extern "C" int hpccg_generate_matrix(int32_t nx, int32_t ny, int32_t nz, int32_t *rowindex,
                                     int32_t *colindex, double *values, double *x, double *b,
                                     double *xexact, int64_t *nnz) {
  if (nx < 1 || ny < 1 || nz < 1 || !rowindex || !colindex || !values || !x || !b || !xexact)
    return HPCCG_ERR_INVALID_ARG;
  const int64_t n = (int64_t)nx * ny * nz;
  if (27 * n > INT32_MAX) return HPCCG_ERR_INVALID_ARG;  // int32 indices, as the reference
  const int64_t plane = (int64_t)nx * ny;
  int64_t cur = 0;  // 0-based write position
  for (int64_t row = 0; row < n; ++row) {
    const int ix = (int)(row % nx) + 1, iy = (int)((row / nx) % ny) + 1, iz = (int)(row / plane) + 1;
    rowindex[row] = (int32_t)(cur + 1);
    const int z0 = iz > 1 ? -1 : 0, z1 = iz < nz ? 1 : 0;
    const int y0 = iy > 1 ? -1 : 0, y1 = iy < ny ? 1 : 0;
    const int x0 = ix > 1 ? -1 : 0, x1 = ix < nx ? 1 : 0;
    const int64_t start = cur;
    for (int sz = z0; sz <= z1; ++sz)
      for (int sy = y0; sy <= y1; ++sy)
        for (int sx = x0; sx <= x1; ++sx) {
          colindex[cur] = (int32_t)(row + 1 + sz * plane + (int64_t)sy * nx + sx);
          values[cur] = (sz | sy | sx) ? -1.0 : 27.0;
          ++cur;
        }
    x[row] = 0.0;
    b[row] = 28.0 - (double)(cur - start);
    xexact[row] = 1.0;
  }
  rowindex[n] = (int32_t)(cur + 1);
  *nnz = cur;
  return HPCCG_OK;
}

extern "C" void hpccg_gpu_destroy(hpccg_ctx *c) {
  if (!c) return;
  release_mixed(c);
  if (c->cg_exec) cudaGraphExecDestroy(c->cg_exec);
  if (c->cg_graph) cudaGraphDestroy(c->cg_graph);
  void *bufs[] = {c->d_rowptr, c->d_col, c->d_val, c->d_ell_col, c->d_ell_val, c->d_r, c->d_p,
                  c->d_Ap, c->d_x, c->d_b, c->d_partials, c->d_counter, c->d_state, c->d_hist};
  for (void *p : bufs)
    if (p) cudaFree(p);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->solve0) cudaEventDestroy(c->solve0);
  if (c->solve1) cudaEventDestroy(c->solve1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

#define HPCCG_TRY(call)                                                      \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      rc = set_cuda_error(e_, #call, __FILE__, __LINE__);                    \
      goto fail;                                                             \
    }                                                                        \
  } while (0)

extern "C" int hpccg_gpu_create(int32_t nrow, int64_t nnz, const int32_t *rowindex,
                                const int32_t *colindex, const double *values, hpccg_ctx **out) {
  if (!out || nrow < 1 || nnz < 0 || nnz > INT32_MAX || !rowindex || (nnz > 0 && (!colindex || !values)))
    return HPCCG_ERR_INVALID_ARG;
  *out = nullptr;
  hpccg_ctx *c = new hpccg_ctx();
  int *d_flags = nullptr;
  int h_flags[2] = {0, 0};
  int rc = init_ctx_common(c);
  if (rc) goto fail;
  if ((rc = alloc_matrix(c, nrow, nnz, 0))) goto fail;
  HPCCG_TRY(cudaMemcpyAsync(c->d_rowptr, rowindex, sizeof(int32_t) * ((size_t)nrow + 1),
                            cudaMemcpyHostToDevice, c->stream));
  if (nnz > 0) {
    HPCCG_TRY(cudaMemcpyAsync(c->d_col, colindex, sizeof(int32_t) * (size_t)nnz,
                              cudaMemcpyHostToDevice, c->stream));
    HPCCG_TRY(cudaMemcpyAsync(c->d_val, values, sizeof(double) * (size_t)nnz,
                              cudaMemcpyHostToDevice, c->stream));
  }
  HPCCG_TRY(cudaMalloc(&d_flags, sizeof(int) * 2));
  HPCCG_TRY(cudaMemsetAsync(d_flags, 0, sizeof(int) * 2, c->stream));
  rebase_kernel<<<grid_for(c, std::max<int64_t>(nnz, (int64_t)nrow + 1)), kBlock, 0, c->stream>>>(
      nrow, nnz, c->d_rowptr, c->d_col, d_flags);
  check_rows_kernel<<<grid_for(c, nrow), kBlock, 0, c->stream>>>(nrow, nnz, c->d_rowptr, 0, d_flags,
                                                                 d_flags + 1);
  HPCCG_TRY(cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 2, cudaMemcpyDeviceToHost, c->stream));
  HPCCG_TRY(cudaStreamSynchronize(c->stream));
  if (h_flags[0]) {
    rc = HPCCG_ERR_INVALID_ARG;
    goto fail;
  }
  c->ell_width = h_flags[1];
  if ((rc = alloc_ell(c))) goto fail;
  if (c->d_ell_col)
    csr_to_ell_kernel<<<grid_for(c, c->npad), kBlock, 0, c->stream>>>(
        nrow, c->d_rowptr, c->d_col, c->d_val, c->d_ell_col, c->d_ell_val, c->npad, c->ell_width);
  HPCCG_TRY(cudaStreamSynchronize(c->stream));
  HPCCG_TRY(cudaGetLastError());
  cudaFree(d_flags);
  *out = c;
  return HPCCG_OK;
fail:
  if (d_flags) cudaFree(d_flags);
  hpccg_gpu_destroy(c);
  return rc ? rc : HPCCG_ERR_CUDA;
}

// Compares row i of the CSR with generate_matrix(nx,ny,nz): the kept
// stencil columns in (sz, sy, sx) order, 27.0 on the diagonal and -1.0
// elsewhere (MPI/src/SparseMatrix.F90:146-159).  Counts rows that differ.
__global__ void check_stencil_kernel(int32_t n, int nx, int ny, int nz, const int32_t *rowptr,
                                     const int32_t *col, const double *val, unsigned *bad) {
  const int nxy = nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int iz = i / nxy, rem = i - iz * nxy, iy = rem / nx, ix = rem - iy * nx;
    const int32_t e = rowptr[i + 1];
    int32_t k = rowptr[i];
    bool ok = k >= 0 && e >= k;
    for (int sz = -1; sz <= 1 && ok; ++sz)
      for (int sy = -1; sy <= 1 && ok; ++sy)
        for (int sx = -1; sx <= 1 && ok; ++sx) {
          if ((unsigned)(iz + sz) >= (unsigned)nz || (unsigned)(iy + sy) >= (unsigned)ny ||
              (unsigned)(ix + sx) >= (unsigned)nx)
            continue;
          const int j = i + sz * nxy + sy * nx + sx;
          ok = k < e && col[k] == j && val[k] == (j == i ? 27.0 : -1.0);
          ++k;
        }
    if (!ok || k != e) atomicAdd(bad, 1u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && rowptr[0] != 0) atomicAdd(bad, 1u);
}

extern "C" int hpccg_gpu_set_geometry(hpccg_ctx *c, int32_t nx, int32_t ny, int32_t nz) {
  if (!c || nx < 1 || ny < 1 || nz < 1 || (int64_t)nx * ny * nz != (int64_t)c->nrow) return HPCCG_ERR_INVALID_ARG;
  c->gx = c->gy = c->gz = 0;
  if (c->spmv_kind == HPCCG_SPMV_STENCIL) {
    c->spmv_kind = HPCCG_SPMV_AUTO;
    c->spmv_tuned = false;
  }
  unsigned *d_bad = nullptr, h_bad = 1;
  HPCCG_CUDA(cudaMalloc(&d_bad, sizeof(unsigned)));
  cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(unsigned), c->stream);
  if (e == cudaSuccess) {
    check_stencil_kernel<<<grid_for(c, c->nrow), kBlock, 0, c->stream>>>(c->nrow, nx, ny, nz, c->d_rowptr,
                                                                         c->d_col, c->d_val, d_bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_bad);
  if (e != cudaSuccess) return set_cuda_error(e, "stencil check", __FILE__, __LINE__);
  if (h_bad) return HPCCG_ERR_UNSUPPORTED;
  c->gx = nx;
  c->gy = ny;
  c->gz = nz;
  // the FP64 TMA walk under the tile map reads p and x through these maps;
  // without them (a map the driver refuses) the same walk runs on plain loads
  c->tmaps_ok = fp64_map(nx, ny, nz, c->num_sms).tiles_x > 0 &&
                make_stencil_tmap64(&c->tmaps[0], c->d_p, nx, ny, nz, kR64BoxX, kR64BoxY) == HPCCG_OK &&
                make_stencil_tmap64(&c->tmaps[1], c->d_x, nx, ny, nz, kR64BoxX, kR64BoxY) == HPCCG_OK;
  c->cg_graph_kind = -1;  // a graph captured before holds the old map
  return HPCCG_OK;
}

// Longest row of generate_matrix: min(n,3) kept offsets per axis.
static int generated_width(int nx, int ny, int nz) {
  return std::min(nx, 3) * std::min(ny, 3) * std::min(nz, 3);
}

extern "C" int hpccg_gpu_create_generated(int32_t nx, int32_t ny, int32_t nz, double *d_x,
                                          double *d_b, double *d_xexact, hpccg_ctx **out) {
  if (!out || nx < 1 || ny < 1 || nz < 1) return HPCCG_ERR_INVALID_ARG;
  const int64_t n = (int64_t)nx * ny * nz;
  if (27 * n > INT32_MAX) return HPCCG_ERR_INVALID_ARG;
  *out = nullptr;
  const int64_t nnz = axis_total(nx) * axis_total(ny) * axis_total(nz);
  const int W = generated_width(nx, ny, nz);
  hpccg_ctx *c = new hpccg_ctx();
  int rc = init_ctx_common(c);
  if (rc) goto fail;
  if ((rc = alloc_matrix(c, (int32_t)n, nnz, W))) goto fail;
  if ((rc = alloc_ell(c))) goto fail;
  generate_kernel<<<grid_for(c, n), kBlock, 0, c->stream>>>(nx, ny, nz, c->d_rowptr, c->d_col, c->d_val,
                                                          c->d_ell_col, c->d_ell_val, c->npad, W,
                                                          d_x, d_b, d_xexact);
  pad_rows_kernel<<<grid_for(c, c->npad - n + 1), kBlock, 0, c->stream>>>((int32_t)n, c->npad, W,
                                                                        c->d_ell_col, c->d_ell_val);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    rc = set_cuda_error(cudaGetLastError(), "generate matrix", __FILE__, __LINE__);
    goto fail;
  }
  if ((rc = hpccg_gpu_set_geometry(c, nx, ny, nz))) goto fail;  // the matrix-free SpMV's precondition
  *out = c;
  return HPCCG_OK;
fail:
  hpccg_gpu_destroy(c);
  return rc ? rc : HPCCG_ERR_CUDA;
}

extern "C" int hpccg_gpu_info(const hpccg_ctx *c, int32_t *nrow, int64_t *nnz, int32_t *ell_width) {
  if (!c) return HPCCG_ERR_INVALID_ARG;
  if (nrow) *nrow = c->nrow;
  if (nnz) *nnz = c->nnz;
  if (ell_width) *ell_width = c->ell_width;
  return HPCCG_OK;
}

__global__ void rebase_up_kernel(int32_t n, int64_t nnz, int32_t *rowptr, int32_t *col) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += stride) rowptr[i] += 1;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += stride) col[j] += 1;
}

extern "C" int hpccg_gpu_download_csr(const hpccg_ctx *c, int32_t *rowindex, int32_t *colindex,
                                      double *values) {
  if (!c || !rowindex || !colindex || !values) return HPCCG_ERR_INVALID_ARG;
  int32_t *tr = nullptr, *tc = nullptr;
  HPCCG_CUDA(cudaMalloc(&tr, sizeof(int32_t) * ((size_t)c->nrow + 1)));
  if (cudaMalloc(&tc, sizeof(int32_t) * std::max<int64_t>(c->nnz, 1)) != cudaSuccess) {
    cudaFree(tr);
    return HPCCG_ERR_OOM;
  }
  cudaMemcpyAsync(tr, c->d_rowptr, sizeof(int32_t) * ((size_t)c->nrow + 1), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(tc, c->d_col, sizeof(int32_t) * (size_t)c->nnz, cudaMemcpyDeviceToDevice, c->stream);
  rebase_up_kernel<<<grid_for(c, std::max<int64_t>(c->nnz, c->nrow + 1)), kBlock, 0, c->stream>>>(c->nrow, c->nnz, tr, tc);
  cudaMemcpyAsync(rowindex, tr, sizeof(int32_t) * ((size_t)c->nrow + 1), cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(colindex, tc, sizeof(int32_t) * (size_t)c->nnz, cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(values, c->d_val, sizeof(double) * (size_t)c->nnz, cudaMemcpyDeviceToHost, c->stream);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  cudaFree(tr);
  cudaFree(tc);
  HPCCG_CUDA(e);
  return HPCCG_OK;
}

// The project's counter-based uniform generator (splitmix64 finaliser).
__global__ void uniform_pm1_kernel(uint64_t seed, int64_t offset, int64_t n, double *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + (uint64_t)(offset + i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * 0x1.0p-53;
    out[i] = 2.0 * u - 1.0;
  }
}

extern "C" int hpccg_gpu_uniform_pm1(hpccg_ctx *c, uint64_t seed, int64_t offset, int64_t n,
                                     double *d_out) {
  if (!c || n < 0 || offset < 0 || (n > 0 && !d_out)) return HPCCG_ERR_INVALID_ARG;
  if (n == 0) return HPCCG_OK;
  uniform_pm1_kernel<<<grid_for(c, n), kBlock, 0, c->stream>>>(seed, offset, n, d_out);
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  return HPCCG_OK;
}
