// hpccg_mixed_fcg.cu -- the learned preconditioner inside mixed precision:
// FP64 iterative refinement around a flexible (Polak-Ribiere) CG whose vectors
// are FP32 and whose preconditioner is the U-Net.
//
// Outer loop, FP64 on the device: r = b - A x with the context's FP64 SpMV
// (reference term order), stop when ||r|| <= rel_tol ||b|| -- the FP64 true
// residual alone decides -- else solve A d = r / ||r|| with the inner
// solver and update x += ||r|| d in FP64.
//
// Inner solver, FP32 vectors (dot products accumulated in FP64): flexible CG
// on the matrix-free operator (28 x - sum of the 3x3x3 box, the FP32 form of
// the generate_matrix stencil) with z = s * net(r / s), s = rms(r); beta =
// r.(z - z_old) / (r.z)_prev.  Plain CG (z = r) takes over when r.z <= 0 or
// the residual stalls (no 10% drop in 5 iterations); u = NULL runs plain CG.
// It stops at ||r_in|| <= max(1e-5, 0.5 rel_tol ||b|| / ||r||) (the inner
// start is scaled to norm 1), the adaptive target of hpccg_gpu_solve_mixed.
//
// The loop is host-driven: each inner iteration reads its scalars back (the
// network application, about 3 ms at 256^3, dominates the time anyway).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>

#include "hpccg_rows.cuh"

struct hpccg_unet;
extern "C" int hpccg_unet_forward_on(hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz, const float *d_in,
                                     float *d_out, cudaStream_t stream);

namespace hpccg {

struct MfcgState {
  double rr64, bb;      // FP64 residual and right-hand side norms squared
  double rz;            // r.z of the current direction (set by the host)
  double rznew, rzold;  // r.z and r.z_old of the latest preconditioner application
  double pAp, rr, alpha, beta, s, scale;
};

struct MfcgArgs {
  int n;
  double *x, *r64;
  const double *b;
  float *r, *p, *Ap, *z, *zold, *d, *nn_in, *nn_out;
  MfcgState *st;
  Reduction red;
  StencilGeom geom;
  PlaneMap pm;  // the FP32 walk's map (four or one column per thread)
};

// FP64 r = b - A x and r.r with the context's FP64 strategy.
template <class S>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_mfcg_residual(const __grid_constant__ SpmvArgs a, MfcgArgs g) {
  __shared__ double smem[32];
  EpiResidual epi{g.b, g.r64};
  const double part = S::rows(a, g.x, epi);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double rr = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->rr64 = rr;
  }
}
__global__ void __launch_bounds__(kBlock) k_mfcg_bnorm(MfcgArgs g) {
  __shared__ double smem[32];
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    a = fma(g.b[i], g.b[i], a);
  const double t = block_sum<kBlock>(a, smem);
  if (arrive_last(g.red, t)) {
    const double v = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->bb = v;
  }
}

// inner start: r = r64 / ||r64|| in FP32, d = 0, z_old = 0
__global__ void k_mfcg_start(MfcgArgs g) {
  const double inv = 1.0 / g.st->scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    g.r[i] = (float)(g.r64[i] * inv);
    g.d[i] = 0.f;
    g.zold[i] = 0.f;
  }
}

// network input r / s
__global__ void k_mfcg_nn_in(MfcgArgs g) {
  const float inv = g.st->s > 0.0 ? (float)(1.0 / g.st->s) : 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    g.nn_in[i] = g.r[i] * inv;
}

// z = s * net(r/s) or z = r; r.z and r.z_old, both reduced in a fixed order
// (r.z_old's block partials sit in the upper half of the scratch)
constexpr int kHalf = kMaxPartials / 2;
__global__ void __launch_bounds__(kBlock) k_mfcg_zdots(MfcgArgs g, int use_net) {
  __shared__ double smem[32];
  const float s = (float)g.st->s;
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const float ri = g.r[i];
    const float zi = use_net ? s * g.nn_out[i] : ri;
    g.z[i] = zi;
    a += (double)(ri * zi);
    b += (double)(ri * g.zold[i]);
  }
  const double ta = block_sum<kBlock>(a, smem);
  const double tb = block_sum<kBlock>(b, smem);
  if (threadIdx.x == 0) g.red.partials[kHalf + blockIdx.x] = tb;  // ordered by arrive_last's fence
  if (arrive_last(g.red, ta)) {
    const double va = finish_sum<kBlock>(g.red, smem);
    double vb = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kBlock)
      vb = __dadd_rn(vb, ((volatile double *)g.red.partials)[kHalf + i]);
    vb = block_sum<kBlock>(vb, smem);
    if (threadIdx.x == 0) {
      g.st->rznew = va;
      g.st->rzold = vb;
    }
  }
}

// p = z + beta p (restart: p = z); z_old = z
__global__ void k_mfcg_update_p(MfcgArgs g, int restart) {
  const float beta = restart ? 0.f : (float)g.st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const float zi = g.z[i];
    g.p[i] = restart ? zi : fmaf(beta, g.p[i], zi);
    g.zold[i] = zi;
  }
}

// Ap = A p in FP32 (matrix-free) and p.Ap
struct EpiAp32 {
  float *y;
  __device__ __forceinline__ double operator()(int i, float s, float pi) const {
    y[i] = s;
    return (double)(pi * s);
  }
  __device__ __forceinline__ double store4(int i, float4 s, float4 pv) const {
    *reinterpret_cast<float4 *>(y + i) = s;
    return (double)(pv.x * s.x + pv.y * s.y + pv.z * s.z + pv.w * s.w);
  }
};
template <bool W4>
__global__ void __launch_bounds__(kBlock) k_mfcg_spmv(MfcgArgs g) {
  __shared__ double smem[32];
  EpiAp32 epi{g.Ap};
  double part;
  if constexpr (W4)
    part = stencil_rows_boxw<4>(g.geom, g.pm, g.p, epi);
  else
    part = stencil_rows_box(g.geom, g.pm, g.p, epi);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double v = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      g.st->pAp = v;
      g.st->alpha = g.st->rz / v;
    }
  }
}

// d += alpha p, r -= alpha Ap, r.r
__global__ void __launch_bounds__(kBlock) k_mfcg_update(MfcgArgs g) {
  __shared__ double smem[32];
  const float alpha = (float)g.st->alpha;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    g.d[i] = fmaf(alpha, g.p[i], g.d[i]);
    const float ri = fmaf(-alpha, g.Ap[i], g.r[i]);
    g.r[i] = ri;
    part += (double)(ri * ri);
  }
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double v = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) g.st->rr = v;
  }
}

// x += scale * d in FP64
__global__ void k_mfcg_end(MfcgArgs g) {
  const double scale = g.st->scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    g.x[i] = fma(scale, (double)g.d[i], g.x[i]);
}

}  // namespace hpccg

using namespace hpccg;

extern "C" int hpccg_gpu_solve_mixed_fcg(hpccg_ctx *c, hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz,
                                         const double *d_b, double *d_x, double rel_tol, int32_t max_outer,
                                         int32_t max_inner, hpccg_mixed_fcg_info *info) {
  if (!c || !d_b || !d_x || !(rel_tol > 0.0) || max_outer < 1 || max_inner < 1) return HPCCG_ERR_INVALID_ARG;
  if ((int64_t)nx * ny * nz != c->nrow) return HPCCG_ERR_INVALID_ARG;
  if (!c->gx || c->gx != nx || c->gy != ny || c->gz != nz) return HPCCG_ERR_UNSUPPORTED;  // matrix-free FP32 operator
  if (u && (nx % 8 || ny % 8 || nz % 8)) return HPCCG_ERR_UNSUPPORTED;  // the U-Net's four levels
  int rc = autotune_spmv(c);
  if (rc) return rc;
  const int n = c->nrow;
  const size_t v4 = sizeof(float) * (size_t)c->npad, bytes = sizeof(double) * (size_t)n;
  float *f32 = nullptr;
  MfcgState *st = nullptr;
  if (cudaMalloc(&f32, 8 * v4) != cudaSuccess || cudaMalloc(&st, sizeof(MfcgState)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(f32);
    return HPCCG_ERR_OOM;
  }
  auto cleanup = [&]() {
    cudaFree(f32);
    cudaFree(st);
  };
  cudaStream_t s = c->stream;
  MfcgArgs g;
  g.n = n;
  g.x = c->d_x;
  g.r64 = c->d_r;
  g.b = c->d_b;
  float *f[8];
  for (int k = 0; k < 8; ++k) f[k] = f32 + (size_t)k * c->npad;
  g.r = f[0], g.p = f[1], g.Ap = f[2], g.z = f[3], g.zold = f[4], g.d = f[5], g.nn_in = f[6], g.nn_out = f[7];
  g.st = st;
  g.red = reduction_of(c);
  g.geom = StencilGeom{nx, ny, nz};
  const PlaneMap q4 = boxw_map(4, nx, ny, nz, (int64_t)c->num_sms * 4 * kBlock);
  const bool w4 = q4.plane > 0 && plane_grid(q4) <= kMaxPartials / 2;
  g.pm = w4 ? q4 : plane_map(nx, ny, nz, kMaxPartials / 2);
  if (!w4 && g.pm.plane <= 0) {
    cleanup();
    return HPCCG_ERR_UNSUPPORTED;
  }
  const int sgrid = plane_grid(g.pm);
  SpmvArgs a = spmv_args(c);
  MfcgState h{};
  auto read_state = [&]() -> int {
    HPCCG_CUDA(cudaMemcpyAsync(&h, st, sizeof(MfcgState), cudaMemcpyDeviceToHost, s));
    HPCCG_CUDA(cudaStreamSynchronize(s));
    return HPCCG_OK;
  };
  auto write_state = [&]() -> int {
    HPCCG_CUDA(cudaMemcpyAsync(st, &h, sizeof(MfcgState), cudaMemcpyHostToDevice, s));
    return HPCCG_OK;
  };
  auto residual = [&]() -> int {
    const int e = dispatch_strategy(a, [&](auto strat) {
      using St = decltype(strat);
      k_mfcg_residual<St><<<St::grid(a, c->grid), kBlock, 0, s>>>(a, g);
      return (int)cudaGetLastError();
    });
    return e ? set_cuda_error((cudaError_t)e, "mixed fcg residual", __FILE__, __LINE__) : read_state();
  };
  if (cudaMemcpyAsync(c->d_b, d_b, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(c->d_x, d_x, bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(st, 0, sizeof(MfcgState), s) != cudaSuccess || cudaEventRecord(c->solve0, s) != cudaSuccess) {
    rc = set_cuda_error(cudaGetLastError(), "mixed fcg set-up", __FILE__, __LINE__);
    cleanup();
    return rc;
  }
  k_mfcg_bnorm<<<c->grid, kBlock, 0, s>>>(g);
  int32_t outer = 0, inner_total = 0, applies = 0, fallback = 0, status = HPCCG_OK;
  if (!(rc = read_state())) rc = residual();
  const double bnorm = sqrt(h.bb);
  double rnorm = sqrt(h.rr64);
  while (!rc && outer < max_outer && rnorm > rel_tol * bnorm) {
    ++outer;
    const double target = std::max(1e-5, 0.5 * rel_tol * bnorm / rnorm);
    h.scale = rnorm;
    if ((rc = write_state())) break;
    k_mfcg_start<<<c->grid, kBlock, 0, s>>>(g);
    bool use_net = u != nullptr, restart = true;
    double rin = 1.0, best = 1.0;
    int since_best = 0;
    for (int k = 0; k < max_inner && rin > target; ++k) {
      h.s = rin / sqrt((double)n);  // rms of the inner residual
      if ((rc = write_state())) break;
      if (use_net) {
        k_mfcg_nn_in<<<c->grid, kBlock, 0, s>>>(g);
        if ((rc = hpccg_unet_forward_on(u, nx, ny, nz, g.nn_in, g.nn_out, s))) break;
        ++applies;
      }
      k_mfcg_zdots<<<c->grid, kBlock, 0, s>>>(g, use_net ? 1 : 0);
      if ((rc = read_state())) break;
      if (use_net && !(h.rznew > 0.0)) {  // the network lost positivity on this residual: plain CG
        use_net = false;
        fallback = 1;
        restart = true;
        k_mfcg_zdots<<<c->grid, kBlock, 0, s>>>(g, 0);
        if ((rc = read_state())) break;
      }
      h.beta = restart ? 0.0 : (h.rznew - h.rzold) / h.rz;  // Polak-Ribiere
      h.rz = h.rznew;
      if ((rc = write_state())) break;
      k_mfcg_update_p<<<c->grid, kBlock, 0, s>>>(g, restart ? 1 : 0);
      restart = false;
      if (w4)
        k_mfcg_spmv<true><<<sgrid, kBlock, 0, s>>>(g);
      else
        k_mfcg_spmv<false><<<sgrid, kBlock, 0, s>>>(g);
      k_mfcg_update<<<c->grid, kBlock, 0, s>>>(g);
      const cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) {
        rc = set_cuda_error(le, "mixed fcg inner", __FILE__, __LINE__);
        break;
      }
      if ((rc = read_state())) break;
      ++inner_total;
      if (!(h.pAp > 0.0) || !isfinite(h.rr)) {
        status = HPCCG_ERR_BREAKDOWN;
        break;
      }
      rin = sqrt(h.rr);
      if (rin < 0.9 * best) {
        best = rin;
        since_best = 0;
      } else if (use_net && ++since_best >= 5) {  // stalled: continue as plain CG
        use_net = false;
        fallback = 1;
        restart = true;
      }
    }
    if (rc || status) break;
    k_mfcg_end<<<c->grid, kBlock, 0, s>>>(g);
    if ((rc = residual())) break;
    rnorm = sqrt(h.rr64);
  }
  cudaEventRecord(c->solve1, s);
  cudaMemcpyAsync(d_x, c->d_x, bytes, cudaMemcpyDeviceToDevice, s);
  cudaStreamSynchronize(s);
  cudaEventElapsedTime(&c->last_solve_ms, c->solve0, c->solve1);
  cleanup();
  if (rc) return rc;
  const double relres = rel_norm(rnorm, bnorm);
  if (info) {
    info->outer_iters = outer;
    info->inner_iters = inner_total;
    info->nn_applies = applies;
    info->fallback = fallback;
    info->status = status;
    info->reserved = 0;
    info->relres = relres;
  }
  if (status) return status;
  return relres <= rel_tol ? HPCCG_OK : HPCCG_ERR_NOT_CONVERGED;
}
