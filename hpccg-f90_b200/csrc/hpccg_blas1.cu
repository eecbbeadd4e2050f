// hpccg_blas1.cu -- op-level drop-ins for MPI/src/vector_operations.F90:40-169.
//
// Element-wise ops use separately rounded multiply and add, so with the same
// scalars they are bit-identical to the reference's loops.  The two dot
// products reduce per thread (strided), per block (fixed butterfly), then over
// the fixed block grid in index order by the last block to arrive: the result
// is reproducible run to run; it differs from the reference's sequential sum
// only by reassociation.  These calls accept any device pointers (no
// alignment assumption) and synchronise before returning, like the
// reference's blocking routines.
#include "hpccg_internal.cuh"

namespace hpccg {

constexpr int kResultSlot = kMaxPartials - 1;

template <bool SQUARE>
__global__ void __launch_bounds__(kBlock) k_dot(int n, const double *__restrict__ x,
                                                const double *__restrict__ y, Reduction red) {
  __shared__ double smem[32];
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double xi = __ldg(x + i);
    part = __dadd_rn(part, __dmul_rn(xi, SQUARE ? xi : __ldg(y + i)));
  }
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(red, tot)) {
    const double v = finish_sum<kBlock>(red, smem);
    if (threadIdx.x == 0) red.partials[kResultSlot] = v;
  }
}

__global__ void k_waxpby(int n, double alpha, const double *__restrict__ x, double beta,
                         const double *__restrict__ y, double *__restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    w[i] = __dadd_rn(__dmul_rn(alpha, x[i]), __dmul_rn(beta, y[i]));
}
__global__ void k_wwpby(int n, double beta, const double *__restrict__ y, double *w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    w[i] = __dadd_rn(w[i], __dmul_rn(beta, y[i]));
}
__global__ void k_wxbw(int n, const double *__restrict__ x, double beta, double *w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    w[i] = __dadd_rn(x[i], __dmul_rn(beta, w[i]));
}
__global__ void k_vcopy(int n, const double *__restrict__ x, double *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i];
}

static int finish(hpccg_ctx *c) {
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  return HPCCG_OK;
}

static int dot(hpccg_ctx *c, int32_t n, const double *x, const double *y, bool square, double *result) {
  if (!c || n < 0 || !x || (!square && !y) || !result) return HPCCG_ERR_INVALID_ARG;
  if (n == 0) {
    *result = 0.0;
    return HPCCG_OK;
  }
  if (square) k_dot<true><<<c->grid, kBlock, 0, c->stream>>>(n, x, x, reduction_of(c));
  else k_dot<false><<<c->grid, kBlock, 0, c->stream>>>(n, x, y, reduction_of(c));
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaMemcpyAsync(result, c->d_partials + kResultSlot, sizeof(double),
                             cudaMemcpyDeviceToHost, c->stream));
  return finish(c);
}

}  // namespace hpccg

using namespace hpccg;

// vector_operations.F90:40-71
extern "C" int hpccg_gpu_ddot(hpccg_ctx *c, int32_t n, const double *d_x, const double *d_y,
                              double *result) {
  return dot(c, n, d_x, d_y, false, result);
}

// vector_operations.F90:73-103
extern "C" int hpccg_gpu_ddot1(hpccg_ctx *c, int32_t n, const double *d_x, double *result) {
  return dot(c, n, d_x, nullptr, true, result);
}

// vector_operations.F90:105-121
extern "C" int hpccg_gpu_waxpby(hpccg_ctx *c, int32_t n, double alpha, const double *d_x,
                                double beta, const double *d_y, double *d_w) {
  if (!c || n < 0 || (n && (!d_x || !d_y || !d_w))) return HPCCG_ERR_INVALID_ARG;
  if (n) k_waxpby<<<c->grid, kBlock, 0, c->stream>>>(n, alpha, d_x, beta, d_y, d_w);
  return finish(c);
}

// vector_operations.F90:123-137
extern "C" int hpccg_gpu_wwpby(hpccg_ctx *c, int32_t n, double beta, const double *d_y, double *d_w) {
  if (!c || n < 0 || (n && (!d_y || !d_w))) return HPCCG_ERR_INVALID_ARG;
  if (n) k_wwpby<<<c->grid, kBlock, 0, c->stream>>>(n, beta, d_y, d_w);
  return finish(c);
}

// vector_operations.F90:139-153
extern "C" int hpccg_gpu_wxbw(hpccg_ctx *c, int32_t n, const double *d_x, double beta, double *d_w) {
  if (!c || n < 0 || (n && (!d_x || !d_w))) return HPCCG_ERR_INVALID_ARG;
  if (n) k_wxbw<<<c->grid, kBlock, 0, c->stream>>>(n, d_x, beta, d_w);
  return finish(c);
}

// vector_operations.F90:155-169
extern "C" int hpccg_gpu_vcopy(hpccg_ctx *c, int32_t n, const double *d_x, double *d_y) {
  if (!c || n < 0 || (n && (!d_x || !d_y))) return HPCCG_ERR_INVALID_ARG;
  if (n) k_vcopy<<<c->grid, kBlock, 0, c->stream>>>(n, d_x, d_y);
  return finish(c);
}
