// hpccg_internal.cuh -- shared device helpers and the context layout.
//
// Device memory layout of one matrix (all on the context's GPU):
//   CSR   rowptr[N+1], col[nnz] (0-based int32), val[nnz] (FP64)  -- boundary copy
//   ELL   col/val column-major [W][Npad], W = max row length, Npad = N rounded up
//         to 128; row i's k-th nonzero sits at k*Npad+i; unused slots hold
//         col = i and val = 0 (they add an exact zero after the row's real terms,
//         so the sum order equals the reference's k order).
//   Scratch: per-block partial sums for deterministic reductions, one arrival
//         counter, the CG scalar state and the residual history.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/hpccg_gpu.h"

namespace hpccg {

constexpr int kBlock = 256;          // threads per block for streaming kernels
constexpr int kMaxPartials = 8192;   // capacity of the partial-sum scratch
constexpr int kEllAlign = 128;       // ELL column stride alignment (rows)

// Scalar state of one CG solve, device resident.  Field names follow the
// reference's local variables in MPI/src/numerics.F90:41-82.
struct CgState {
  double rtrans, oldrtrans, normr, alpha, beta, pAp, rr_last, tolerance;
  int k;          // iteration being executed (reference loop variable)
  int max_iter;
  int niters;
  int status;     // HPCCG_OK or HPCCG_ERR_BREAKDOWN
  int x_pending;  // 1 while x += alpha*p of the previous iteration is deferred
  int cont;       // 1 while the loop continues (mirrors the graph condition)
  int pad[2];
};

struct Reduction {
  double *partials;   // [kMaxPartials]
  unsigned *counter;  // arrival counter, reset by the last block
};

// ||r|| / ||b|| from the two norms.  A non-finite b (a NaN anywhere in it)
// gives NaN, so a solver reports it instead of taking it for convergence; for
// b = 0 the ratio is 0 when r = 0 too and the largest double otherwise (the
// relative target can then never be met).
__host__ __device__ __forceinline__ double rel_norm(double rnorm, double bnorm) {
  if (bnorm > 0.0) return rnorm / bnorm;
  if (bnorm == 0.0) return rnorm == 0.0 ? 0.0 : (rnorm > 0.0 ? 1.7976931348623157e308 : rnorm);
  return bnorm;  // NaN
}
// The same from the squared norms r.r and b.b.
__host__ __device__ __forceinline__ double rel_residual(double rr, double bb) {
  return rel_norm(sqrt(rr), sqrt(bb));
}

}  // namespace hpccg

struct hpccg_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  int32_t nrow = 0;
  int64_t nnz = 0;
  int32_t npad = 0;
  int32_t ell_width = 0;
  // CSR (0-based)
  int32_t *d_rowptr = nullptr;
  int32_t *d_col = nullptr;
  double *d_val = nullptr;
  // ELL
  int32_t *d_ell_col = nullptr;
  double *d_ell_val = nullptr;
  // CG work vectors and staging
  double *d_r = nullptr, *d_p = nullptr, *d_Ap = nullptr, *d_x = nullptr, *d_b = nullptr;
  // scratch
  double *d_partials = nullptr;
  unsigned *d_counter = nullptr;
  hpccg::CgState *d_state = nullptr;
  double *d_hist = nullptr;
  int32_t hist_cap = 0;
  int grid = 0;  // blocks for streaming kernels (multiple of the SM count)
  // grid of generate_matrix the CSR was checked against (0: unknown)
  int32_t gx = 0, gy = 0, gz = 0;
  // tensor maps of d_p and d_x for the FP64 TMA walk (tmaps_ok false: plain loads)
  CUtensorMap tmaps[2];
  bool tmaps_ok = false;
  // SpMV selection
  int spmv_kind = HPCCG_SPMV_AUTO;
  int spmv_param = 0;
  bool mixed_fused_off = false;  // hpccg_gpu_set_mixed_fused(ctx, 0)
  bool spmv_tuned = false;
  // CG graph
  cudaGraph_t cg_graph = nullptr;
  cudaGraphExec_t cg_exec = nullptr;
  int cg_graph_kind = -1, cg_graph_param = -1;
  int32_t cg_graph_hist_cap = 0;
  // events for timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t solve0 = nullptr, solve1 = nullptr;
  float last_solve_ms = 0.f;
};

namespace hpccg {

// ---- error plumbing -------------------------------------------------------
int set_cuda_error(cudaError_t e, const char *what, const char *file, int line);

#define HPCCG_CUDA(call)                                                    \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) return ::hpccg::set_cuda_error(e_, #call, __FILE__, __LINE__); \
  } while (0)

// ---- deterministic reductions --------------------------------------------
// Warp butterfly then a fixed-order pass over the warp sums: the result only
// depends on the block's inputs, not on scheduling.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double *smem) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = (lane < BLOCK / 32) ? smem[lane] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

// Writes this block's partial and returns true in exactly one thread of the
// last block to arrive; that thread then sums partials[0..gridDim.x) in index
// order, so the total is identical on every run.
__device__ __forceinline__ bool arrive_last(const Reduction &red, double block_total) {
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    red.partials[blockIdx.x] = block_total;
    __threadfence();
    const unsigned prev = atomicAdd(red.counter, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  return s_last;
}

// Fixed-order sum of the partials by the whole last block (stride pattern is
// fixed, so the association order is fixed).  Resets the counter.
template <int BLOCK>
__device__ __forceinline__ double finish_sum(const Reduction &red, double *smem) {
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += BLOCK)
    v = __dadd_rn(v, ((volatile double *)red.partials)[i]);
  v = block_sum<BLOCK>(v, smem);
  if (threadIdx.x == 0) *red.counter = 0u;
  return v;
}

inline Reduction reduction_of(const hpccg_ctx *c) { return Reduction{c->d_partials, c->d_counter}; }

// ---- kernel launchers shared between translation units --------------------
int launch_spmv(hpccg_ctx *c, const double *x, double *y, cudaStream_t s);
int autotune_spmv(hpccg_ctx *c);
int ensure_workspace(hpccg_ctx *c, int32_t hist_cap);
void release_mixed(const hpccg_ctx *c);

}  // namespace hpccg
