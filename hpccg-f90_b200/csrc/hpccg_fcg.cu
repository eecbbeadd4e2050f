// hpccg_fcg.cu -- flexible (Polak-Ribiere) preconditioned CG with the U-Net as
// the preconditioner.  Vectors, dots and the convergence test are FP64; the
// preconditioner M(r) = s * net(r / s), s = rms(r), runs in BF16/FP32 on the
// tensor cores.  Plain CG is the fallback (z = r) when the preconditioned
// iteration stalls or loses positivity, and the FP64 true residual b - A x
// decides convergence.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>

#include "hpccg_rows.cuh"

struct hpccg_unet;
extern "C" int hpccg_unet_forward_on(hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz, const float *d_in,
                                     float *d_out, cudaStream_t stream);

namespace hpccg {

struct FcgState {
  double rr, pAp, rz, rz_old_new, rz_new, alpha, beta, s, bb;
};

struct FcgArgs {
  int n;
  double *x, *r, *p, *Ap, *z, *zold;
  const double *b;
  float *nn_in, *nn_out;
  FcgState *st;
  Reduction red;
};

template <class S>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_fcg_spmv_dot(const __grid_constant__ SpmvArgs a, FcgArgs g) {
  __shared__ double smem[32];
  EpiDot epi{g.p, g.Ap};
  const double part = S::rows(a, g.p, epi);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double pAp = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      g.st->pAp = pAp;
      g.st->alpha = g.st->rz / pAp;
    }
  }
}

template <class S>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_fcg_residual(const __grid_constant__ SpmvArgs a, FcgArgs g) {
  __shared__ double smem[32];
  EpiResidual epi{g.b, g.r};
  const double part = S::rows(a, g.x, epi);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double rr = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->rr = rr;
  }
}

// x += alpha p, r -= alpha Ap, rr = r.r
__global__ void __launch_bounds__(kBlock) k_fcg_update(FcgArgs g) {
  __shared__ double smem[32];
  const double alpha = g.st->alpha;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    g.x[i] = fma(alpha, g.p[i], g.x[i]);
    const double ri = fma(-alpha, g.Ap[i], g.r[i]);
    g.r[i] = ri;
    part = fma(ri, ri, part);
  }
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double rr = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->rr = rr;
  }
}

// Network input: r / s with s = rms(r).
__global__ void k_fcg_nn_in(FcgArgs g) {
  const double s = g.st->s;
  const double inv = s > 0.0 ? 1.0 / s : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    g.nn_in[i] = (float)(g.r[i] * inv);
}

// z = s * net(r/s) (use_net) or z = r (plain CG), and r.z.
__global__ void __launch_bounds__(kBlock) k_fcg_zdots(FcgArgs g, int use_net) {
  __shared__ double smem[32];
  const double s = g.st->s;
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const double zi = use_net ? s * (double)g.nn_out[i] : g.r[i];
    g.z[i] = zi;
    a = fma(g.r[i], zi, a);
  }
  const double ta = block_sum<kBlock>(a, smem);
  if (arrive_last(g.red, ta)) {
    const double v = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->rz_new = v;
  }
}

// b.b
__global__ void __launch_bounds__(kBlock) k_fcg_bnorm(FcgArgs g) {
  __shared__ double smem[32];
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) a = fma(g.b[i], g.b[i], a);
  const double ta = block_sum<kBlock>(a, smem);
  if (arrive_last(g.red, ta)) {
    const double v = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->bb = v;
  }
}

// r.zold (zold = the previous preconditioned residual)
__global__ void __launch_bounds__(kBlock) k_fcg_dot_old(FcgArgs g) {
  __shared__ double smem[32];
  double b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    b = fma(g.r[i], g.zold[i], b);
  const double tb = block_sum<kBlock>(b, smem);
  if (arrive_last(g.red, tb)) {
    const double v = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->rz_old_new = v;
  }
}

// p = z + beta p ; zold = z
__global__ void k_fcg_update_p(FcgArgs g, int restart) {
  const double beta = restart ? 0.0 : g.st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const double zi = g.z[i];
    g.p[i] = restart ? zi : fma(beta, g.p[i], zi);
    g.zold[i] = zi;
  }
}

}  // namespace hpccg

using namespace hpccg;

struct FcgRes {
  double *z = nullptr, *zold = nullptr;
  float *nn_in = nullptr, *nn_out = nullptr;
  FcgState *st = nullptr;
};

extern "C" int hpccg_gpu_solve_fcg(hpccg_ctx *c, hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz,
                                   const double *d_b, double *d_x, double rel_tol, int32_t max_iter,
                                   hpccg_fcg_info *info) {
  if (!c || !d_b || !d_x || !(rel_tol > 0.0) || max_iter < 1) return HPCCG_ERR_INVALID_ARG;
  if ((int64_t)nx * ny * nz != c->nrow) return HPCCG_ERR_INVALID_ARG;
  int rc = autotune_spmv(c);
  if (rc) return rc;
  const int n = c->nrow;
  const size_t v8 = sizeof(double) * (size_t)c->npad, v4 = sizeof(float) * (size_t)c->npad;
  FcgRes R;
  HPCCG_CUDA(cudaMalloc(&R.z, v8));
  HPCCG_CUDA(cudaMalloc(&R.zold, v8));
  HPCCG_CUDA(cudaMalloc(&R.nn_in, v4));
  HPCCG_CUDA(cudaMalloc(&R.nn_out, v4));
  HPCCG_CUDA(cudaMalloc(&R.st, sizeof(FcgState)));
  auto cleanup = [&]() {
    cudaFree(R.z);
    cudaFree(R.zold);
    cudaFree(R.nn_in);
    cudaFree(R.nn_out);
    cudaFree(R.st);
  };
  cudaStream_t s = c->stream;
  const size_t bytes = sizeof(double) * (size_t)n;
  FcgArgs g;
  g.n = n;
  g.x = c->d_x;
  g.r = c->d_r;
  g.p = c->d_p;
  g.Ap = c->d_Ap;
  g.b = c->d_b;
  g.z = R.z;
  g.zold = R.zold;
  g.nn_in = R.nn_in;
  g.nn_out = R.nn_out;
  g.st = R.st;
  g.red = reduction_of(c);
  const SpmvArgs a = spmv_args(c);
  cudaMemcpyAsync(c->d_b, d_b, bytes, cudaMemcpyDeviceToDevice, s);
  cudaMemcpyAsync(c->d_x, d_x, bytes, cudaMemcpyDeviceToDevice, s);
  cudaMemsetAsync(R.zold, 0, v8, s);
  cudaMemsetAsync(R.st, 0, sizeof(FcgState), s);
  HPCCG_CUDA(cudaEventRecord(c->solve0, s));
  FcgState h;
  auto read_state = [&]() -> int {
    HPCCG_CUDA(cudaMemcpyAsync(&h, R.st, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
    HPCCG_CUDA(cudaStreamSynchronize(s));
    return HPCCG_OK;
  };
  auto residual = [&]() -> int {
    return dispatch_strategy(a, [&](auto strat) {
      using St = decltype(strat);
      k_fcg_residual<St><<<St::grid(a, c->grid), kBlock, 0, s>>>(a, g);
      return (int)cudaGetLastError();
    });
  };
  int32_t iters = 0, applies = 0, fallback = 0, status = HPCCG_OK;
  double relres = 0.0;
  k_fcg_bnorm<<<c->grid, kBlock, 0, s>>>(g);
  if ((rc = read_state())) {
    cleanup();
    return rc;
  }
  const double bnorm = sqrt(h.bb);
  const double tol = rel_tol * bnorm;
  // preconditioner application on r: z (and r.z, r.zold)
  auto precond = [&](bool use_net) -> int {
    if (use_net && u) {
      HPCCG_CUDA(cudaMemcpyAsync(&R.st->s, &h.s, sizeof(double), cudaMemcpyHostToDevice, s));
      k_fcg_nn_in<<<c->grid, kBlock, 0, s>>>(g);
      int e = hpccg_unet_forward_on(u, nx, ny, nz, R.nn_in, R.nn_out, s);
      if (e) return e;
      ++applies;
    }
    k_fcg_zdots<<<c->grid, kBlock, 0, s>>>(g, use_net && u ? 1 : 0);
    k_fcg_dot_old<<<c->grid, kBlock, 0, s>>>(g);
    HPCCG_CUDA(cudaGetLastError());
    return read_state();
  };
  bool use_net = u != nullptr;
  const bool trace = getenv("HPCCG_FCG_TRACE") != nullptr;
  rc = residual();
  if (!rc) rc = read_state();
  double rnorm = sqrt(h.rr);
  double best = rnorm;
  int since_best = 0;
  bool restart = true;
  for (iters = 0; !rc && iters < max_iter && rnorm > tol;) {
    h.s = rnorm / sqrt((double)n);
    if ((rc = precond(use_net))) break;
    double rz = h.rz_new;
    if (use_net && !(rz > 0.0)) {  // preconditioner lost positivity on this residual: fall back
      use_net = false;
      fallback = 1;
      if ((rc = precond(false))) break;
      rz = h.rz_new;
      restart = true;
    }
    // Polak-Ribiere beta = r.(z - zold) / rz_prev
    const double beta = restart ? 0.0 : (rz - h.rz_old_new) / h.rz;
    h.beta = beta;
    h.rz = rz;
    HPCCG_CUDA(cudaMemcpyAsync(R.st, &h, sizeof(FcgState), cudaMemcpyHostToDevice, s));
    k_fcg_update_p<<<c->grid, kBlock, 0, s>>>(g, restart ? 1 : 0);
    restart = false;
    rc = dispatch_strategy(a, [&](auto strat) {
      using St = decltype(strat);
      k_fcg_spmv_dot<St><<<St::grid(a, c->grid), kBlock, 0, s>>>(a, g);
      return (int)cudaGetLastError();
    });
    if (rc) break;
    k_fcg_update<<<c->grid, kBlock, 0, s>>>(g);
    if ((rc = read_state())) break;
    ++iters;
    if (!(h.pAp > 0.0) || !isfinite(h.rr)) {
      status = HPCCG_ERR_BREAKDOWN;
      break;
    }
    rnorm = sqrt(h.rr);
    if (trace)
      fprintf(stderr, "fcg it %d relres %.3e rz %.3e beta %.3e pAp %.3e net %d\n", iters, rnorm / bnorm, rz, beta,
              h.pAp, use_net ? 1 : 0);
    if (rnorm < 0.9 * best) {
      best = rnorm;
      since_best = 0;
    } else if (use_net && ++since_best >= 5) {  // stalled: continue as plain CG
      use_net = false;
      fallback = 1;
      restart = true;
    }
    if (rnorm <= tol) {  // the FP64 true residual decides
      if ((rc = residual()) || (rc = read_state())) break;
      rnorm = sqrt(h.rr);
      restart = true;
    }
  }
  if (!rc) {
    if ((rc = residual()) == 0) rc = read_state();
  }
  relres = rel_norm(sqrt(h.rr), bnorm);
  HPCCG_CUDA(cudaEventRecord(c->solve1, s));
  cudaMemcpyAsync(d_x, c->d_x, bytes, cudaMemcpyDeviceToDevice, s);
  cudaStreamSynchronize(s);
  cudaEventElapsedTime(&c->last_solve_ms, c->solve0, c->solve1);
  cleanup();
  if (rc) return rc > 0 && rc < 16 ? rc : set_cuda_error((cudaError_t)rc, "fcg", __FILE__, __LINE__);
  if (info) {
    info->iters = iters;
    info->nn_applies = applies;
    info->fallback = fallback;
    info->status = status;
    info->relres = relres;
  }
  if (status) return status;
  return relres <= rel_tol ? HPCCG_OK : HPCCG_ERR_NOT_CONVERGED;
}
