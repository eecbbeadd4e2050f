// hpccg_mixed.cu -- FP64 iterative refinement around an FP32 / BF16-value inner CG.
//
// Outer loop (FP64, on the device):  r = b - A x (FP64 values, the bit-exact
// reference SpMV), stop when ||r|| <= rel_tol ||b||; otherwise solve A d = r/||r||
// approximately with the inner CG and update x += ||r|| d in FP64.
// Inner CG (FP32 vectors; FP32 or BF16 copies of A's values; FP32 row sums;
// FP64 dot-product accumulation) stops at ||r_in|| <= target ||r_in,0|| where
// target = inner_rtol, or adaptively max(floor, 0.5 rel_tol ||b|| / ||r||).
// The FP64 true residual decides: the solve only reports success when
// the FP64 residual meets rel_tol.
//
// One CUDA graph: bnorm, residual64, while(outer){ start_inner,
// while(inner){ P, A, B }, end_inner, residual64 }.
#include <stdlib.h>

#include <algorithm>
#include <type_traits>

#include <cudaTypedefs.h>

#include <mutex>

#include "hpccg_rows.cuh"
#include "hpccg_rows_lp.cuh"
#include "hpccg_iter_tma.cuh"
#include "hpccg_stencil_tma.cuh"

namespace hpccg {

struct MixedState {
  double bb, rr64, scale, rel_tol, relres, target, inner_rtol, inner_floor;
  double rtrans, rr0, alpha, beta;
  double pAp, rAp, ApAp;  // dots of the last fused pass
  int outer, max_outer, inner_k, max_inner, inner_total, status, pending, inner_break;
  int cont_outer, cont_inner;
  int passes;  // fused passes run in this inner solve (selects the r, p buffers)
  int pad;
};

struct MixedArgs {
  int n, npad;
  const double *b;
  double *x, *r64;
  float *r, *p, *Ap, *d;
  const int32_t *ell_col;
  const void *val_lp;
  MixedState *st;
  Reduction red;
  StencilGeom geom;  // matrix-free inner SpMV when the context uses the stencil
  PlaneMap pm;
  cudaGraphConditionalHandle cond_outer, cond_inner;
  int use_cond;
  int skip_done;  // fused pass: return at once when the inner solve has ended
};

__device__ __forceinline__ void set_outer(const MixedArgs &g, int v) {
  g.st->cont_outer = v;
  if (g.use_cond) cudaGraphSetConditional(g.cond_outer, (unsigned)v);
}
__device__ __forceinline__ void set_inner(const MixedArgs &g, int v) {
  g.st->cont_inner = v;
  if (g.use_cond) cudaGraphSetConditional(g.cond_inner, (unsigned)v);
}

__global__ void __launch_bounds__(kBlock) k_mp_bnorm(MixedArgs g) {
  __shared__ double smem[32];
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const double bi = g.b[i];
    part = __dadd_rn(part, __dmul_rn(bi, bi));
  }
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double bb = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      g.st->bb = bb;
      g.st->outer = 0;
      g.st->inner_total = 0;
      g.st->status = HPCCG_OK;
    }
  }
}

// r64 = b - A x64 (FP64, reference order) and the outer decision.
template <class S>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_mp_residual64(const __grid_constant__ SpmvArgs a, MixedArgs g) {
  __shared__ double smem[32];
  EpiResidual epi{g.b, g.r64};
  const double part = S::rows(a, g.x, epi);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double rr = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      MixedState &st = *g.st;
      st.rr64 = rr;
      st.relres = rel_residual(rr, st.bb);
      int cont = (st.relres > st.rel_tol) && (st.outer < st.max_outer);
      if (!isfinite(st.relres)) {
        st.status = HPCCG_ERR_BREAKDOWN;
        cont = 0;
      }
      if (cont) {
        st.scale = sqrt(rr);
        st.target = st.inner_rtol > 0.0 ? st.inner_rtol
                                        : fmax(st.inner_floor, 0.5 * st.rel_tol / st.relres);
        st.outer += 1;
      }
      set_outer(g, cont);
    }
  }
}

// The refinement residual of the fused inner iteration: r = b - A x in FP64,
// stored unscaled in FP32 (the first fused pass scales it by 1/||r||), its
// norm and the outer decision; with FIRST also b.b (the solve's first call).
struct EpiResidualF {
  const double *b;
  float *r;
  double bb;
  __device__ __forceinline__ double operator()(int i, double s) {
    const double bi = __ldg(b + i);
    bb = __dadd_rn(bb, __dmul_rn(bi, bi));
    const double ri = __dsub_rn(bi, s);
    r[i] = (float)ri;
    return __dmul_rn(ri, ri);
  }
  __device__ __forceinline__ double operator()(int i, double s, double) { return (*this)(i, s); }
};
// Four rows at once (i a multiple of 4): b from shared memory, r by one 16-byte store.
template <bool FIRST>
struct EpiResidualF4 {
  float *r;
  double bb;
  __device__ __forceinline__ double store4(int i, const double y[4], const double *b4) {
    const double2 b01 = *reinterpret_cast<const double2 *>(b4);
    const double2 b23 = *reinterpret_cast<const double2 *>(b4 + 2);
    const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
    float4 ro;
    double rr = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (FIRST) bb = __dadd_rn(bb, __dmul_rn(bv[k], bv[k]));
      const double rk = __dsub_rn(bv[k], y[k]);
      reinterpret_cast<float *>(&ro)[k] = (float)rk;
      rr = __dadd_rn(rr, __dmul_rn(rk, rk));
    }
    *reinterpret_cast<float4 *>(r + i) = ro;
    return rr;
  }
};

// The outer decision of the fused refinement from v[0] = r.r (and v[1] = b.b
// on the first call); thread 0 of the last block.
template <bool FIRST>
__device__ __forceinline__ void residual_decision(const MixedArgs &g, const double v[4]) {
  MixedState &st = *g.st;
  if (FIRST) {
    st.bb = v[1];
    st.outer = 0;
    st.inner_total = 0;
    if (st.status != HPCCG_ERR_TIMEOUT) st.status = HPCCG_OK;  // a TMA walk's expired wait stands
  }
  const double rr = v[0];
  st.rr64 = rr;
  st.relres = rel_residual(rr, st.bb);
  int cont = !st.status && (st.relres > st.rel_tol) && (st.outer < st.max_outer);
  if (!isfinite(st.relres)) {
    st.status = HPCCG_ERR_BREAKDOWN;
    cont = 0;
  }
  if (cont) {
    st.scale = sqrt(rr);
    st.target = st.inner_rtol > 0.0 ? st.inner_rtol : fmax(st.inner_floor, 0.5 * st.rel_tol / st.relres);
    st.outer += 1;
  }
  set_outer(g, cont);
}

template <class S, bool FIRST>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_mp_residual_f(const __grid_constant__ SpmvArgs a, MixedArgs g) {
  __shared__ double smem[4 * 32];
  EpiResidualF epi{g.b, g.r, 0.0};
  double v[4] = {S::rows(a, g.x, epi), 0.0, 0.0, 0.0};
  v[1] = epi.bb;
  if (reduce4_last<kBlock>(g.red, v, smem) && threadIdx.x == 0) residual_decision<FIRST>(g, v);
}

// The same with x streamed by TMA (stencil_rows_tma64box; t: 32 x 64 tiles).
template <bool FIRST>
__global__ void __launch_bounds__(kBlock, 2) k_mp_residual_tma(MixedArgs g, TmaTile t,
                                                               const __grid_constant__ CUtensorMap xmap,
                                                               const __grid_constant__ CUtensorMap bmap) {
  __shared__ double smem[4 * 32];
  EpiResidualF4<FIRST> epi{g.r, 0.0};
  double v[4] = {stencil_rows_tma64box(t, &xmap, &bmap, epi, &g.st->status), 0.0, 0.0, 0.0};
  v[1] = epi.bb;
  if (reduce4_last<kBlock>(g.red, v, smem) && threadIdx.x == 0) residual_decision<FIRST>(g, v);
}

// Start of an inner solve of the fused iteration: scalar state only (the
// first pass scales r, clears d and forms rr0).
__global__ void k_mp_start_inner_f(MixedArgs g) {
  if (threadIdx.x == 0) {
    MixedState &st = *g.st;
    st.inner_k = 0;
    st.pending = 0;
    st.inner_break = 0;
    st.passes = 0;
    set_inner(g, st.rr64 > 0.0 && st.max_inner > 0);
  }
}

// r32 = r64 / ||r64||, d = 0, rr0 = ||r32||^2.
__global__ void __launch_bounds__(kBlock) k_mp_start_inner(MixedArgs g) {
  __shared__ double smem[32];
  const double inv = 1.0 / g.st->scale;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const float ri = (float)(g.r64[i] * inv);
    g.r[i] = ri;
    g.d[i] = 0.f;
    part += (double)ri * (double)ri;
  }
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double rr = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      MixedState &st = *g.st;
      st.rtrans = rr;
      st.rr0 = rr;
      st.inner_k = 0;
      st.pending = 0;
      st.inner_break = 0;
      st.passes = 0;
      set_inner(g, rr > 0.0 && st.max_inner > 0);
    }
  }
}

// p = r (first) or d += alpha p (deferred), p = r + beta p.
__global__ void __launch_bounds__(kBlock) k_mp_update_p(MixedArgs g) {
  const MixedState *st = g.st;
  const int n4 = g.n >> 2;
  const int stride = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  float4 *p4 = reinterpret_cast<float4 *>(g.p);
  const float4 *r4 = reinterpret_cast<const float4 *>(g.r);
  float4 *d4 = reinterpret_cast<float4 *>(g.d);
  if (st->inner_k == 0) {
    for (int i = tid; i < n4; i += stride) p4[i] = __ldcs(r4 + i);
    for (int i = 4 * n4 + tid; i < g.n; i += stride) g.p[i] = g.r[i];
    return;
  }
  const float alpha = (float)st->alpha, beta = (float)st->beta;
  const int pend = st->pending;
  for (int i = tid; i < n4; i += stride) {
    float4 pi = p4[i];
    const float4 ri = __ldcs(r4 + i);
    if (pend) {
      float4 di = __ldcs(d4 + i);
      di.x = fmaf(alpha, pi.x, di.x);
      di.y = fmaf(alpha, pi.y, di.y);
      di.z = fmaf(alpha, pi.z, di.z);
      di.w = fmaf(alpha, pi.w, di.w);
      __stcs(d4 + i, di);
    }
    pi.x = fmaf(beta, pi.x, ri.x);
    pi.y = fmaf(beta, pi.y, ri.y);
    pi.z = fmaf(beta, pi.z, ri.z);
    pi.w = fmaf(beta, pi.w, ri.w);
    p4[i] = pi;
  }
  for (int i = 4 * n4 + tid; i < g.n; i += stride) {
    const float pi = g.p[i];
    if (pend) g.d[i] = fmaf(alpha, pi, g.d[i]);
    g.p[i] = fmaf(beta, pi, g.r[i]);
  }
}

struct EpiDot32 {
  const float *p;
  float *y;
  __device__ __forceinline__ double operator()(int i, float s) const {
    y[i] = s;
    return (double)__ldg(p + i) * (double)s;
  }
  // pi = p[i], already at hand in the matrix-free walk
  __device__ __forceinline__ double operator()(int i, float s, float pi) const {
    y[i] = s;
    return (double)pi * (double)s;
  }
  // rows i .. i+3 (i a multiple of 4)
  __device__ __forceinline__ double store4(int i, float4 s, float4 pi) const {
    *reinterpret_cast<float4 *>(y + i) = s;
    return ((double)pi.x * s.x + (double)pi.y * s.y) + ((double)pi.z * s.z + (double)pi.w * s.w);
  }
};

// Ap = A p with low-precision values, alpha = rtrans / p.Ap.
template <class S, typename VT>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_mp_spmv_dot(MixedArgs g) {
  __shared__ double smem[32];
  EpiDot32 epi{g.p, g.Ap};
  const double part = S::rows(g.n, g.npad, g.ell_col, reinterpret_cast<const VT *>(g.val_lp), g.p, epi, g.geom, g.pm);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double pAp = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      MixedState &st = *g.st;
      st.pending = 0;
      const double alpha = st.rtrans / pAp;
      if (!(pAp > 0.0) || !isfinite(alpha)) {
        st.inner_break = 1;
        st.alpha = 0.0;
      } else {
        st.alpha = alpha;
      }
    }
  }
}

// The same with the matrix-free SpMV fed by TMA (hpccg_stencil_tma.cuh).
__global__ void __launch_bounds__(kBlock) k_mp_spmv_dot_tma(MixedArgs g, TmaTile t,
                                                            const __grid_constant__ CUtensorMap map) {
  __shared__ double smem[32];
  EpiDot32 epi{g.p, g.Ap};
  const double part = stencil_rows_tma(t, &map, epi, &g.st->status);
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double pAp = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      MixedState &st = *g.st;
      st.pending = 0;
      const double alpha = st.rtrans / pAp;
      if (!(pAp > 0.0) || !isfinite(alpha)) {
        st.inner_break = 1;
        st.alpha = 0.0;
      } else {
        st.alpha = alpha;
      }
    }
  }
}

// r -= alpha Ap, rr, inner stop test.
__global__ void __launch_bounds__(kBlock) k_mp_update_r(MixedArgs g) {
  __shared__ double smem[32];
  if (g.st->inner_break) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_inner(g, 0);
    return;
  }
  const float nalpha = -(float)g.st->alpha;
  const int n4 = g.n >> 2;
  const int stride = gridDim.x * blockDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  float4 *r4 = reinterpret_cast<float4 *>(g.r);
  const float4 *a4 = reinterpret_cast<const float4 *>(g.Ap);
  double part = 0.0;
  for (int i = tid; i < n4; i += stride) {
    float4 ri = r4[i];
    const float4 ai = __ldcs(a4 + i);
    ri.x = fmaf(nalpha, ai.x, ri.x);
    ri.y = fmaf(nalpha, ai.y, ri.y);
    ri.z = fmaf(nalpha, ai.z, ri.z);
    ri.w = fmaf(nalpha, ai.w, ri.w);
    r4[i] = ri;
    part += (double)ri.x * ri.x + (double)ri.y * ri.y + (double)ri.z * ri.z + (double)ri.w * ri.w;
  }
  for (int i = 4 * n4 + tid; i < g.n; i += stride) {
    const float ri = fmaf(nalpha, g.Ap[i], g.r[i]);
    g.r[i] = ri;
    part += (double)ri * ri;
  }
  const double tot = block_sum<kBlock>(part, smem);
  if (arrive_last(g.red, tot)) {
    const double rr = finish_sum<kBlock>(g.red, smem);
    if (threadIdx.x == 0) {
      MixedState &st = *g.st;
      st.inner_k += 1;
      st.inner_total += 1;
      st.pending = 1;
      st.beta = rr / st.rtrans;
      st.rtrans = rr;
      const int cont = isfinite(rr) && (rr > st.target * st.target * st.rr0) && (st.inner_k < st.max_inner);
      set_inner(g, cont);
    }
  }
}

// d += alpha p (pending), x64 += ||r64|| d.
__global__ void __launch_bounds__(kBlock) k_mp_end_inner(MixedArgs g) {
  const MixedState *st = g.st;
  const int pend = st->pending;
  const float alpha = (float)st->alpha;
  const double scale = st->scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const float di = pend ? fmaf(alpha, g.p[i], g.d[i]) : g.d[i];
    g.x[i] = fma(scale, (double)di, g.x[i]);
  }
}

// One fused pass of the matrix-free inner CG (hpccg_iter_tma.cuh).  Pass k
// reads r and p from buffers k & 1 and writes buffers (k + 1) & 1; p0, p1
// (box 72 x 68), r0, r1 (box 72 x 66) and dm (box 64 x 64, of g.d) are the
// tensor maps of the buffers.
struct IterBufs {
  float *r[2], *p[2];
};
__global__ void __launch_bounds__(kItBlock, 1) k_mp_iter_tma(MixedArgs g, TmaTile t, IterBufs b,
                                                          const __grid_constant__ CUtensorMap p0,
                                                          const __grid_constant__ CUtensorMap p1,
                                                          const __grid_constant__ CUtensorMap r0,
                                                          const __grid_constant__ CUtensorMap r1,
                                                          const __grid_constant__ CUtensorMap dm) {
  __shared__ double smem[4 * 32];
  MixedState *st = g.st;
  // a pass of an unrolled loop body after the inner solve has ended does nothing
  // (cont_inner changes only in the last block of a pass, after every block has read it)
  if (g.skip_done && !st->cont_inner) return;
  const int par = st->passes & 1;
  const bool first = st->passes == 0;
  IterScalars sc;
  sc.alpha = (float)st->alpha;
  sc.nalpha = -sc.alpha;
  sc.beta = (float)st->beta;
  sc.inv = first ? (float)(1.0 / st->scale) : 1.f;
  double v[4];
  if (first)
    iter_rows_tma<true>(t, &p0, &r0, &dm, b.r[1], b.p[1], g.d, sc, v, &st->status);
  else
    iter_rows_tma<false>(t, par ? &p1 : &p0, par ? &r1 : &r0, &dm, b.r[par ^ 1], b.p[par ^ 1], g.d, sc, v,
                         &st->status);
  if (reduce4_last<kItBlock>(g.red, v, smem) && threadIdx.x == 0) {
    const double pAp = v[0], rAp = v[1], ApAp = v[2], rr = v[3];
    st->pAp = pAp;
    st->rAp = rAp;
    st->ApAp = ApAp;
    if (!first) {
      st->inner_k += 1;
      st->inner_total += 1;
    }
    st->passes += 1;
    st->pending = 0;
    st->rtrans = rr;
    if (first) st->rr0 = rr;
    int cont = isfinite(rr) && (rr > st->target * st->target * st->rr0) && (st->inner_k < st->max_inner);
    const double alpha = rr / pAp;
    if (cont && (!(pAp > 0.0) || !isfinite(alpha))) {
      st->inner_break = 1;
      cont = 0;
    }
    if (cont) {
      // ||r - alpha Ap||^2 for the next beta
      const double rr1 = fma(alpha, fma(alpha, ApAp, -2.0 * rAp), rr);
      st->alpha = alpha;
      st->beta = fmax(rr1, 0.0) / rr;
    }
    set_inner(g, cont);
  }
}

// Plain low-precision y = A x for tests and timing.
struct EpiStore32 {
  float *y;
  __device__ __forceinline__ double operator()(int i, float s, float = 0.f) const {
    y[i] = s;
    return 0.0;
  }
  __device__ __forceinline__ double store4(int i, float4 s, float4) const {
    *reinterpret_cast<float4 *>(y + i) = s;
    return 0.0;
  }
};
template <class S, typename VT>
__global__ void __launch_bounds__(kBlock, S::kMinBlocks) k_spmv_lp(int n, int npad, const int32_t *col,
                                                                   const VT *val, const float *x, float *y,
                                                                   StencilGeom geom, PlaneMap pm) {
  EpiStore32 epi{y};
  S::rows(n, npad, col, val, x, epi, geom, pm);
}

__global__ void __launch_bounds__(kBlock) k_spmv_lp_tma(TmaTile t, const __grid_constant__ CUtensorMap map, float *y,
                                                        int *status) {
  EpiStore32 epi{y};
  stencil_rows_tma(t, &map, epi, status);
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::mutex g_encode_mu;

// A 3D tensor map over a grid vector of `esize`-byte elements, box box_x x box_y x 1;
// out-of-grid elements of a box read as zeros.
static int encode_grid_tmap(CUtensorMap *map, CUtensorMapDataType type, int esize, const void *base, int nx, int ny,
                            int nz, int box_x, int box_y) {
  {
    std::lock_guard<std::mutex> lk(g_encode_mu);
    if (!g_encode) {
      void *fn = nullptr;
      cudaDriverEntryPointQueryResult q;
      const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
      if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return set_cuda_error(e == cudaSuccess ? cudaErrorNotSupported : e, "cuTensorMapEncodeTiled", __FILE__,
                              __LINE__);
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
  }
  // 16-byte base, row and plane strides; 16-byte inner box extent
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((int64_t)nx * esize) % 16 || ((int64_t)box_x * esize) % 16)
    return HPCCG_ERR_UNSUPPORTED;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * esize, (cuuint64_t)nx * ny * esize};
  const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = g_encode(map, type, 3, const_cast<void *>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HPCCG_OK : HPCCG_ERR_UNSUPPORTED;
}

int make_stencil_tmap(CUtensorMap *map, const float *base, int nx, int ny, int nz, int box_y, int box_x) {
  return encode_grid_tmap(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, nx, ny, nz, box_x, box_y);
}

int make_stencil_tmap64(CUtensorMap *map, const double *base, int nx, int ny, int nz, int box_x, int box_y) {
  return encode_grid_tmap(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, base, nx, ny, nz, box_x, box_y);
}

// Plan of the TMA SpMV for a context (nzc = 0: not usable).
static TmaTile tma_plan(const hpccg_ctx *c) {
  // the attribute is per device: set it for the context's device every time
  if (cudaFuncSetAttribute(k_mp_spmv_dot_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaRingBytes) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_spmv_lp_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmaRingBytes) !=
          cudaSuccess) {
    cudaGetLastError();
    return TmaTile{c->gx, c->gy, c->gz, 0, 0, 0, 0};  // not usable: the register walk runs instead
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mp_spmv_dot_tma, kBlock, kTmaRingBytes) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return tma_tile_plan(c->gx, c->gy, c->gz, c->num_sms * per_sm);
}

// Plan of the fused one-pass iteration (nzc = 0: not usable).
static TmaTile iter_plan(const hpccg_ctx *c) {
  const TmaTile none{c->gx, c->gy, c->gz, 0, 0, 0, 0};
  if (cudaFuncSetAttribute(k_mp_iter_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kItSmemBytes) != cudaSuccess) {
    cudaGetLastError();
    return none;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mp_iter_tma, kItBlock, kItSmemBytes) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    return none;
  }
  const TmaTile t = tma_tile_plan(c->gx, c->gy, c->gz, c->num_sms * per_sm, kItTileX, kItTileY);
  // the refinement residual of the fused path reduces four values per block too
  const PlaneMap q = boxw_map(4, c->gx, c->gy, c->gz, (int64_t)c->num_sms * StratStencilBox64::kMinBlocks * kBlock);
  if (q.plane <= 0 || plane_grid(q) > kItMaxGrid) return none;
  return tma_tile_grid(t) <= kItMaxGrid ? t : none;
}

// Plan of the TMA refinement residual (nzc = 0: not usable): 32 x 64 tiles,
// two CTAs per SM in one wave.
static TmaTile residual_plan(const hpccg_ctx *c) {
  if (cudaFuncSetAttribute(k_mp_residual_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kB64RingBytes) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_mp_residual_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kB64RingBytes) !=
          cudaSuccess) {
    cudaGetLastError();
    return TmaTile{c->gx, c->gy, c->gz, 0, 0, 0, 0};
  }
  TmaTile t = tma_tile_plan(c->gx, c->gy, c->gz, 2 * c->num_sms, kB64TileX, kB64TileY);
  if (tma_tile_grid(t) > kItMaxGrid) t.nzc = 0;  // four partials per CTA
  return t;
}

__global__ void k_to_lp(const double *src, float *f32, __nv_bfloat16 *b16, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const double v = src[i];
    if (f32) f32[i] = (float)v;
    if (b16) b16[i] = __double2bfloat16(v);
  }
}

// Low-precision strategy dispatch: the matrix-free stencil when the context
// uses it, else value type by precision, RPT and MINB by param.
template <class F>
inline int dispatch_lp(bool stencil, int precision, int rpt, F &&f) {
  if (stencil) return f(StratLpStencil{}, (float *)nullptr);
  if (precision == 1) {
    switch (rpt) {
      case 1: return f(StratLp<float, 1, 4>{}, (float *)nullptr);
      case 4: return f(StratLp<float, 4, 2>{}, (float *)nullptr);
      default: return f(StratLp<float, 2, 2>{}, (float *)nullptr);
    }
  }
  switch (rpt) {
    case 1: return f(StratLp<__nv_bfloat16, 1, 4>{}, (__nv_bfloat16 *)nullptr);
    case 2: return f(StratLp<__nv_bfloat16, 2, 2>{}, (__nv_bfloat16 *)nullptr);
    default: return f(StratLp<__nv_bfloat16, 4, 2>{}, (__nv_bfloat16 *)nullptr);
  }
}

}  // namespace hpccg

using namespace hpccg;

// Per-context mixed-precision resources, kept beside the context.
struct MixedRes {
  float *r = nullptr, *p = nullptr, *Ap = nullptr, *d = nullptr, *x32 = nullptr, *y32 = nullptr;
  float *val32 = nullptr;
  __nv_bfloat16 *val16 = nullptr;
  int32_t *col27 = nullptr;  // ELL columns padded to width 27 when the FP64 ELL is narrower
  MixedState *st = nullptr;
  cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
  int exec_rpt[3] = {0, 0, 0};
  bool exec_stencil[3] = {false, false, false};
  int rpt[3] = {0, 2, 4};  // rows per thread per precision (index 1 = FP32, 2 = BF16)
  // matrix-free SpMV on p by TMA (when the context uses the stencil and nx % 4 == 0)
  CUtensorMap pmap;
  TmaTile tile{};
  bool tma = false;
  int tma_gx = 0;  // grid the map was made for
  // the fused one-pass iteration: second r and p buffers, maps of p0, p1, r0, r1
  float *r2 = nullptr, *p2 = nullptr;
  CUtensorMap itmap[5];  // p0, p1, r0, r1 and d
  TmaTile itile{};
  bool iter = false;
  // the FP64 refinement residual of the fused iteration with x and b by TMA
  CUtensorMap xmap64, bmap64;
  TmaTile rtile{};
  bool res_tma = false;
  bool exec_fused[3] = {false, false, false};
};

#include <map>
#include <mutex>
static std::mutex g_mixed_mu;
static std::map<const hpccg_ctx *, MixedRes *> g_mixed;

namespace hpccg {
void release_mixed(const hpccg_ctx *c) {
  std::lock_guard<std::mutex> lk(g_mixed_mu);
  auto it = g_mixed.find(c);
  if (it == g_mixed.end()) return;
  MixedRes *m = it->second;
  for (auto &e : m->exec)
    if (e) cudaGraphExecDestroy(e);
  void *bufs[] = {m->r, m->p, m->Ap, m->d, m->x32, m->y32, m->val32, m->val16, m->col27, m->st, m->r2, m->p2};
  for (void *b : bufs)
    if (b) cudaFree(b);
  delete m;
  g_mixed.erase(it);
}
}  // namespace hpccg

__global__ void k_pad_cols27(const int32_t *src, int W, int npad, int32_t *dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)npad; i += (size_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 27; ++k) dst[(size_t)k * npad + i] = k < W ? src[(size_t)k * npad + i] : (int32_t)i;
}
__global__ void k_pad_vals27(const double *src, int W, int npad, double *dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)npad; i += (size_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 27; ++k) dst[(size_t)k * npad + i] = k < W ? src[(size_t)k * npad + i] : 0.0;
}

static bool uses_stencil(const hpccg_ctx *c) { return spmv_args(c).kind == HPCCG_SPMV_STENCIL; }

// Row map of the low-precision matrix-free SpMV: four columns per thread in one
// wave of resident threads (StratLpStencil: 256 threads x 4 blocks per SM) when
// nx allows it, else the context's plane map.
static PlaneMap lp_map(const hpccg_ctx *c) {
  // the FP32 one-column walk takes one line a thread
  const PlaneMap pm = c->gx ? plane_map(c->gx, c->gy, c->gz, kMaxPartials) : spmv_args(c).pm;
  if (!uses_stencil(c) || pm.plane <= 0) return pm;
  const PlaneMap q = boxw_map(4, c->gx, c->gy, c->gz, (int64_t)c->num_sms * StratLpStencil::kMinBlocks * kBlock);
  return q.plane > 0 ? q : pm;
}

static int mixed_res(hpccg_ctx *c, int precision, MixedRes **out) {
  const bool stencil = uses_stencil(c);
  if (!stencil && (!c->d_ell_col || c->ell_width > 27)) return HPCCG_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_mixed_mu);
  MixedRes *&m = g_mixed[c];
  if (!m) {
    m = new MixedRes();
    const size_t vec = sizeof(float) * (size_t)c->npad;
    HPCCG_CUDA(cudaMalloc(&m->r, vec));
    HPCCG_CUDA(cudaMalloc(&m->p, vec));
    HPCCG_CUDA(cudaMalloc(&m->Ap, vec));
    HPCCG_CUDA(cudaMalloc(&m->d, vec));
    HPCCG_CUDA(cudaMemsetAsync(m->p, 0, vec, c->stream));
    HPCCG_CUDA(cudaMalloc(&m->st, sizeof(MixedState)));
  }
  const size_t slots = (size_t)27 * c->npad;
  const double *src = c->d_ell_val;
  double *tmp = nullptr;
  if (!stencil &&
      ((precision == 1 && !m->val32) || (precision == 2 && !m->val16) || (!m->col27 && c->ell_width != 27))) {
    if (c->ell_width != 27) {
      HPCCG_CUDA(cudaMalloc(&tmp, sizeof(double) * slots));
      k_pad_vals27<<<c->num_sms * 8, kBlock, 0, c->stream>>>(c->d_ell_val, c->ell_width, c->npad, tmp);
      src = tmp;
      if (!m->col27) {
        HPCCG_CUDA(cudaMalloc(&m->col27, sizeof(int32_t) * slots));
        k_pad_cols27<<<c->num_sms * 8, kBlock, 0, c->stream>>>(c->d_ell_col, c->ell_width, c->npad, m->col27);
      }
    }
    if (precision == 1 && !m->val32) {
      HPCCG_CUDA(cudaMalloc(&m->val32, sizeof(float) * slots));
      k_to_lp<<<c->num_sms * 8, kBlock, 0, c->stream>>>(src, m->val32, nullptr, slots);
    }
    if (precision == 2 && !m->val16) {
      HPCCG_CUDA(cudaMalloc(&m->val16, sizeof(__nv_bfloat16) * slots));
      k_to_lp<<<c->num_sms * 8, kBlock, 0, c->stream>>>(src, nullptr, m->val16, slots);
    }
    HPCCG_CUDA(cudaStreamSynchronize(c->stream));
    if (tmp) cudaFree(tmp);
    HPCCG_CUDA(cudaGetLastError());
  }
  if (stencil && m->tma_gx != c->gx) {
    m->tile = tma_plan(c);
    m->tma = m->tile.nzc > 0 && make_stencil_tmap(&m->pmap, m->p, c->gx, c->gy, c->gz) == HPCCG_OK;
    m->itile = iter_plan(c);
    m->iter = false;
    if (m->itile.nzc > 0) {
      const size_t vec = sizeof(float) * (size_t)c->npad;
      if (!m->r2) {
        HPCCG_CUDA(cudaMalloc(&m->r2, vec));
        HPCCG_CUDA(cudaMemsetAsync(m->r2, 0, vec, c->stream));
      }
      if (!m->p2) {
        HPCCG_CUDA(cudaMalloc(&m->p2, vec));
        HPCCG_CUDA(cudaMemsetAsync(m->p2, 0, vec, c->stream));
      }
      m->iter = make_stencil_tmap(&m->itmap[0], m->p, c->gx, c->gy, c->gz, kItPBoxY, kItBoxX) == HPCCG_OK &&
                make_stencil_tmap(&m->itmap[1], m->p2, c->gx, c->gy, c->gz, kItPBoxY, kItBoxX) == HPCCG_OK &&
                make_stencil_tmap(&m->itmap[2], m->r, c->gx, c->gy, c->gz, kItRBoxY, kItBoxX) == HPCCG_OK &&
                make_stencil_tmap(&m->itmap[3], m->r2, c->gx, c->gy, c->gz, kItRBoxY, kItBoxX) == HPCCG_OK &&
                make_stencil_tmap(&m->itmap[4], m->d, c->gx, c->gy, c->gz, kItTileY, kItTileX) == HPCCG_OK;
    }
    m->rtile = residual_plan(c);
    m->res_tma = m->rtile.nzc > 0 &&
                 make_stencil_tmap64(&m->xmap64, c->d_x, c->gx, c->gy, c->gz, kB64BoxX, kB64BoxY) == HPCCG_OK &&
                 make_stencil_tmap64(&m->bmap64, c->d_b, c->gx, c->gy, c->gz, kB64TileX, kB64TileY) == HPCCG_OK;
    m->tma_gx = c->gx;
  }
  *out = m;
  return HPCCG_OK;
}

static bool use_tma(const hpccg_ctx *c, const MixedRes *m) { return uses_stencil(c) && m->tma; }
static bool use_iter(const hpccg_ctx *c, const MixedRes *m) {
  return uses_stencil(c) && m->iter && !c->mixed_fused_off;
}

static void launch_iter(hpccg_ctx *c, MixedRes *m, const MixedArgs &g, cudaStream_t s) {
  const IterBufs b{{m->r, m->r2}, {m->p, m->p2}};
  k_mp_iter_tma<<<tma_tile_grid(m->itile), kItBlock, kItSmemBytes, s>>>(g, m->itile, b, m->itmap[0], m->itmap[1],
                                                                      m->itmap[2], m->itmap[3], m->itmap[4]);
}

static MixedArgs mixed_args(hpccg_ctx *c, MixedRes *m, int precision) {
  MixedArgs g{};
  g.n = c->nrow;
  g.npad = c->npad;
  g.b = c->d_b;
  g.x = c->d_x;
  g.r64 = c->d_r;
  g.r = m->r;
  g.p = m->p;
  g.Ap = m->Ap;
  g.d = m->d;
  g.ell_col = m->col27 ? m->col27 : c->d_ell_col;
  g.val_lp = precision == 1 ? (const void *)m->val32 : (const void *)m->val16;
  g.st = m->st;
  g.red = reduction_of(c);
  g.geom = StencilGeom{c->gx, c->gy, c->gz};
  g.pm = lp_map(c);
  return g;
}

// Fused passes per inner-loop body: the while node's per-iteration cost is paid
// once per kInnerUnroll passes; passes after the solve has ended return at once.
#ifndef HPCCG_INNER_UNROLL
#define HPCCG_INNER_UNROLL 4
#endif
constexpr int kInnerUnroll = HPCCG_INNER_UNROLL;

static int launch_inner_body(hpccg_ctx *c, MixedRes *m, int precision, const MixedArgs &g, cudaStream_t s) {
  if (use_iter(c, m)) {
    MixedArgs gs = g;
    gs.skip_done = 1;
    for (int k = 0; k < kInnerUnroll; ++k) launch_iter(c, m, k ? gs : g, s);
    return (int)cudaGetLastError();
  }
  k_mp_update_p<<<c->grid, kBlock, 0, s>>>(g);
  if (use_tma(c, m)) {
    k_mp_spmv_dot_tma<<<tma_tile_grid(m->tile), kBlock, kTmaRingBytes, s>>>(g, m->tile, m->pmap);
    k_mp_update_r<<<c->grid, kBlock, 0, s>>>(g);
    return (int)cudaGetLastError();
  }
  int rc = dispatch_lp(uses_stencil(c), precision, m->rpt[precision], [&](auto strat, auto *vt) {
    using St = decltype(strat);
    using VT = std::remove_pointer_t<decltype(vt)>;
    k_mp_spmv_dot<St, VT><<<St::grid(g.pm, g.geom, c->grid), kBlock, 0, s>>>(g);
    return (int)cudaGetLastError();
  });
  if (rc) return rc;
  k_mp_update_r<<<c->grid, kBlock, 0, s>>>(g);
  return (int)cudaGetLastError();
}

// The refinement residual of the fused iteration (FIRST: also b.b).
static int launch_residual_f(hpccg_ctx *c, const MixedRes *m, const MixedArgs &g, cudaStream_t s, bool first) {
  if (m->res_tma && g.x == c->d_x && g.b == c->d_b) {
    const int grid = tma_tile_grid(m->rtile);
    if (first)
      k_mp_residual_tma<true><<<grid, kBlock, kB64RingBytes, s>>>(g, m->rtile, m->xmap64, m->bmap64);
    else
      k_mp_residual_tma<false><<<grid, kBlock, kB64RingBytes, s>>>(g, m->rtile, m->xmap64, m->bmap64);
    return (int)cudaGetLastError();
  }
  SpmvArgs a = spmv_args(c);
  auto go = [&](auto strat) {
    using St = decltype(strat);
    const int grid = St::grid(a, c->grid);
    if (grid > kItMaxGrid) return (int)HPCCG_ERR_UNSUPPORTED;
    if (first)
      k_mp_residual_f<St, true><<<grid, kBlock, 0, s>>>(a, g);
    else
      k_mp_residual_f<St, false><<<grid, kBlock, 0, s>>>(a, g);
    return (int)cudaGetLastError();
  };
  const PlaneMap q = boxw_map(4, c->gx, c->gy, c->gz, (int64_t)c->num_sms * StratStencilBox64::kMinBlocks * kBlock);
  if (q.plane <= 0) return HPCCG_ERR_UNSUPPORTED;  // iter_plan admits only grids where this map exists
  a.pm = q;
  return go(StratStencilBox64{});
}

static int launch_residual64(hpccg_ctx *c, const MixedArgs &g, cudaStream_t s) {
  SpmvArgs a = spmv_args(c);
  if (a.kind == HPCCG_SPMV_STENCIL) {  // the FP64 box walk, four columns per thread
    const PlaneMap q = boxw_map(4, c->gx, c->gy, c->gz, (int64_t)c->num_sms * StratStencilBox64::kMinBlocks * kBlock);
    if (q.plane > 0) {
      a.pm = q;
      k_mp_residual64<StratStencilBox64><<<StratStencilBox64::grid(a, c->grid), kBlock, 0, s>>>(a, g);
      return (int)cudaGetLastError();
    }
  }
  return dispatch_strategy(a, [&](auto strat) {
    using St = decltype(strat);
    k_mp_residual64<St><<<St::grid(a, c->grid), kBlock, 0, s>>>(a, g);
    return (int)cudaGetLastError();
  });
}

// Adds a while node at the capture point of `s` and captures `body` into it.
template <class Body>
static cudaError_t capture_while(cudaStream_t s, cudaGraphConditionalHandle h, Body &&body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
  if (e != cudaSuccess) return e;
  cudaStream_t bs = nullptr;
  e = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  cudaGraph_t bg = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(bs, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const cudaError_t e1 = body(bs, bg);
    const cudaError_t e2 = cudaStreamEndCapture(bs, &bg);
    e = e1 != cudaSuccess ? e1 : e2;
  }
  cudaStreamDestroy(bs);
  if (e != cudaSuccess) return e;
  return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

static int build_mixed_graph(hpccg_ctx *c, MixedRes *m, int precision) {
  if (m->exec[precision]) {
    cudaGraphExecDestroy(m->exec[precision]);
    m->exec[precision] = nullptr;
  }
  cudaStream_t s = c->stream;
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  cudaGraphConditionalHandle ho = 0;
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&ho, g, 0, cudaGraphCondAssignDefault);
  MixedArgs ga = mixed_args(c, m, precision);
  ga.cond_outer = ho;
  ga.use_cond = 1;
  const bool fused = use_iter(c, m);
  if (e == cudaSuccess) {
    if (fused) {
      e = (cudaError_t)launch_residual_f(c, m, ga, s, true);
    } else {
      k_mp_bnorm<<<c->grid, kBlock, 0, s>>>(ga);
      e = (cudaError_t)launch_residual64(c, ga, s);
    }
  }
  if (e == cudaSuccess)
    e = capture_while(s, ho, [&](cudaStream_t os, cudaGraph_t og) -> cudaError_t {
      cudaGraphConditionalHandle hi = 0;
      cudaError_t ee = cudaGraphConditionalHandleCreate(&hi, og, 0, 0);
      if (ee != cudaSuccess) return ee;
      MixedArgs gi = ga;
      gi.cond_inner = hi;
      if (fused)
        k_mp_start_inner_f<<<1, 32, 0, os>>>(gi);
      else
        k_mp_start_inner<<<c->grid, kBlock, 0, os>>>(gi);
      ee = cudaGetLastError();
      if (ee == cudaSuccess)
        ee = capture_while(os, hi, [&](cudaStream_t is, cudaGraph_t) -> cudaError_t {
          return (cudaError_t)launch_inner_body(c, m, precision, gi, is);
        });
      if (ee == cudaSuccess) {
        k_mp_end_inner<<<c->grid, kBlock, 0, os>>>(gi);
        ee = cudaGetLastError();
      }
      if (ee == cudaSuccess)
        ee = (cudaError_t)(fused ? launch_residual_f(c, m, gi, os, false) : launch_residual64(c, gi, os));
      return ee;
    });
  cudaGraph_t out = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(s, &out);
  if (e == cudaSuccess) e = ee;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&m->exec[precision], out, 0);
  if (out) cudaGraphDestroy(out);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_cuda_error(e, "build mixed graph", __FILE__, __LINE__);
  }
  m->exec_rpt[precision] = m->rpt[precision];
  m->exec_stencil[precision] = uses_stencil(c);
  m->exec_fused[precision] = use_iter(c, m);
  return HPCCG_OK;
}

static int run_mixed_eager(hpccg_ctx *c, MixedRes *m, int precision) {
  MixedArgs g = mixed_args(c, m, precision);
  g.use_cond = 0;
  const bool fused = use_iter(c, m);
  int rc;
  if (fused) {
    rc = launch_residual_f(c, m, g, c->stream, true);
  } else {
    k_mp_bnorm<<<c->grid, kBlock, 0, c->stream>>>(g);
    rc = launch_residual64(c, g, c->stream);
  }
  if (rc) return set_cuda_error((cudaError_t)rc, "residual64", __FILE__, __LINE__);
  for (;;) {
    int cont = 0;
    HPCCG_CUDA(cudaMemcpyAsync(&cont, &m->st->cont_outer, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    HPCCG_CUDA(cudaStreamSynchronize(c->stream));
    if (!cont) break;
    if (fused)
      k_mp_start_inner_f<<<1, 32, 0, c->stream>>>(g);
    else
      k_mp_start_inner<<<c->grid, kBlock, 0, c->stream>>>(g);
    for (;;) {
      int ci = 0;
      HPCCG_CUDA(cudaMemcpyAsync(&ci, &m->st->cont_inner, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      HPCCG_CUDA(cudaStreamSynchronize(c->stream));
      if (!ci) break;
      rc = launch_inner_body(c, m, precision, g, c->stream);
      if (rc) return set_cuda_error((cudaError_t)rc, "inner", __FILE__, __LINE__);
    }
    k_mp_end_inner<<<c->grid, kBlock, 0, c->stream>>>(g);
    rc = fused ? launch_residual_f(c, m, g, c->stream, false) : launch_residual64(c, g, c->stream);
    if (rc) return set_cuda_error((cudaError_t)rc, "residual64", __FILE__, __LINE__);
  }
  return HPCCG_OK;
}

extern "C" int hpccg_gpu_set_mixed_rows_per_thread(hpccg_ctx *c, int32_t precision, int32_t rpt) {
  if (!c || (precision != HPCCG_PREC_FP32 && precision != HPCCG_PREC_BF16)) return HPCCG_ERR_INVALID_ARG;
  if (rpt != 1 && rpt != 2 && rpt != 4) return HPCCG_ERR_INVALID_ARG;
  MixedRes *m = nullptr;
  int rc = mixed_res(c, precision, &m);
  if (rc) return rc;
  m->rpt[precision] = rpt;
  return HPCCG_OK;
}

static int solve_mixed_common(hpccg_ctx *c, int precision, double rel_tol, int32_t max_outer,
                              int32_t max_inner, double inner_rtol, hpccg_mixed_info *info) {
  MixedRes *m = nullptr;
  int rc = mixed_res(c, precision, &m);
  if (rc) return rc;
  if ((rc = autotune_spmv(c))) return rc;
  MixedState h0 = {};
  h0.rel_tol = rel_tol;
  h0.max_outer = max_outer;
  h0.max_inner = max_inner;
  h0.inner_rtol = inner_rtol;
  h0.inner_floor = 1e-5;
  HPCCG_CUDA(cudaMemcpyAsync(m->st, &h0, sizeof(MixedState), cudaMemcpyHostToDevice, c->stream));
  HPCCG_CUDA(cudaEventRecord(c->solve0, c->stream));
  const bool eager = getenv("HPCCG_EAGER") && atoi(getenv("HPCCG_EAGER")) != 0;
  if (eager) {
    if ((rc = run_mixed_eager(c, m, precision))) return rc;
  } else {
    if (!m->exec[precision] || m->exec_rpt[precision] != m->rpt[precision] ||
        m->exec_stencil[precision] != uses_stencil(c) || m->exec_fused[precision] != use_iter(c, m))
      if ((rc = build_mixed_graph(c, m, precision))) return rc;
    HPCCG_CUDA(cudaGraphLaunch(m->exec[precision], c->stream));
  }
  HPCCG_CUDA(cudaEventRecord(c->solve1, c->stream));
  MixedState hs;
  HPCCG_CUDA(cudaMemcpyAsync(&hs, m->st, sizeof(MixedState), cudaMemcpyDeviceToHost, c->stream));
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  HPCCG_CUDA(cudaEventElapsedTime(&c->last_solve_ms, c->solve0, c->solve1));
  if (info) {
    info->outer_iters = hs.outer;
    info->inner_iters = hs.inner_total;
    info->relres = hs.relres;
    info->status = hs.status;
  }
  if (hs.status) return hs.status;
  return hs.relres <= rel_tol ? HPCCG_OK : HPCCG_ERR_NOT_CONVERGED;
}

static bool prec_ok(int p) { return p == HPCCG_PREC_FP32 || p == HPCCG_PREC_BF16; }

extern "C" int hpccg_gpu_solve_mixed_device(hpccg_ctx *c, const double *d_b, double *d_x, int32_t precision,
                                            double rel_tol, int32_t max_outer, int32_t max_inner,
                                            double inner_rtol, hpccg_mixed_info *info) {
  if (!c || !d_b || !d_x || !prec_ok(precision) || !(rel_tol >= 0.0) || max_outer < 0 || max_inner < 0 ||
      !(inner_rtol >= 0.0) || inner_rtol >= 1.0)
    return HPCCG_ERR_INVALID_ARG;
  const size_t bytes = sizeof(double) * (size_t)c->nrow;
  HPCCG_CUDA(cudaMemcpyAsync(c->d_b, d_b, bytes, cudaMemcpyDeviceToDevice, c->stream));
  HPCCG_CUDA(cudaMemcpyAsync(c->d_x, d_x, bytes, cudaMemcpyDeviceToDevice, c->stream));
  const int rc = solve_mixed_common(c, precision, rel_tol, max_outer, max_inner, inner_rtol, info);
  if (rc != HPCCG_OK && rc != HPCCG_ERR_NOT_CONVERGED && rc != HPCCG_ERR_BREAKDOWN) return rc;
  HPCCG_CUDA(cudaMemcpyAsync(d_x, c->d_x, bytes, cudaMemcpyDeviceToDevice, c->stream));
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  return rc;
}

extern "C" int hpccg_gpu_solve_mixed(hpccg_ctx *c, const double *b, double *x, int32_t precision,
                                     double rel_tol, int32_t max_outer, int32_t max_inner, double inner_rtol,
                                     hpccg_mixed_info *info) {
  if (!c || !b || !x || !prec_ok(precision) || !(rel_tol >= 0.0) || max_outer < 0 || max_inner < 0 ||
      !(inner_rtol >= 0.0) || inner_rtol >= 1.0)
    return HPCCG_ERR_INVALID_ARG;
  const size_t bytes = sizeof(double) * (size_t)c->nrow;
  HPCCG_CUDA(cudaMemcpyAsync(c->d_b, b, bytes, cudaMemcpyHostToDevice, c->stream));
  HPCCG_CUDA(cudaMemcpyAsync(c->d_x, x, bytes, cudaMemcpyHostToDevice, c->stream));
  const int rc = solve_mixed_common(c, precision, rel_tol, max_outer, max_inner, inner_rtol, info);
  if (rc != HPCCG_OK && rc != HPCCG_ERR_NOT_CONVERGED && rc != HPCCG_ERR_BREAKDOWN) return rc;
  HPCCG_CUDA(cudaMemcpyAsync(x, c->d_x, bytes, cudaMemcpyDeviceToHost, c->stream));
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  return rc;
}

extern "C" int hpccg_gpu_spmv_lowp(hpccg_ctx *c, int32_t precision, const float *d_x, float *d_y) {
  if (!c || !prec_ok(precision) || !d_x || !d_y || d_x == d_y) return HPCCG_ERR_INVALID_ARG;
  MixedRes *m = nullptr;
  int rc = mixed_res(c, precision, &m);
  if (rc) return rc;
  if (use_tma(c, m)) {
    CUtensorMap xmap;
    if (make_stencil_tmap(&xmap, d_x, c->gx, c->gy, c->gz) == HPCCG_OK) {
      HPCCG_CUDA(cudaMemsetAsync(&m->st->status, 0, sizeof(int), c->stream));
      k_spmv_lp_tma<<<tma_tile_grid(m->tile), kBlock, kTmaRingBytes, c->stream>>>(m->tile, xmap, d_y, &m->st->status);
      HPCCG_CUDA(cudaGetLastError());
      int status = 0;
      HPCCG_CUDA(cudaMemcpyAsync(&status, &m->st->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      HPCCG_CUDA(cudaStreamSynchronize(c->stream));
      return status ? status : HPCCG_OK;
    }
  }
  const int32_t *col = m->col27 ? m->col27 : c->d_ell_col;
  const void *val = precision == 1 ? (const void *)m->val32 : (const void *)m->val16;
  rc = dispatch_lp(uses_stencil(c), precision, m->rpt[precision], [&](auto strat, auto *vt) {
    using St = decltype(strat);
    using VT = std::remove_pointer_t<decltype(vt)>;
    const PlaneMap pm = lp_map(c);
    k_spmv_lp<St, VT><<<St::grid(pm, StencilGeom{c->gx, c->gy, c->gz}, c->grid), kBlock, 0, c->stream>>>(c->nrow, c->npad, col, (const VT *)val, d_x,
                                                                        d_y, StencilGeom{c->gx, c->gy, c->gz}, pm);
    return (int)cudaGetLastError();
  });
  if (rc) return set_cuda_error((cudaError_t)rc, "spmv_lowp", __FILE__, __LINE__);
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_gpu_time_mixed_kernels(hpccg_ctx *c, int32_t precision, int32_t reps, float *ms) {
  if (!c || !prec_ok(precision) || reps < 1 || !ms) return HPCCG_ERR_INVALID_ARG;
  MixedRes *m = nullptr;
  int rc = mixed_res(c, precision, &m);
  if (rc) return rc;
  const size_t vec = sizeof(float) * (size_t)c->npad;
  HPCCG_CUDA(cudaMemsetAsync(m->p, 0, vec, c->stream));
  HPCCG_CUDA(cudaMemsetAsync(m->r, 0, vec, c->stream));
  HPCCG_CUDA(cudaMemsetAsync(m->d, 0, vec, c->stream));
  MixedState h0 = {};
  h0.inner_k = 1;
  h0.rtrans = 1.0;
  h0.alpha = 0.5;
  h0.beta = 0.5;
  h0.pending = 1;
  h0.max_inner = 1 << 30;
  h0.rr0 = 1.0;
  HPCCG_CUDA(cudaMemcpyAsync(m->st, &h0, sizeof(MixedState), cudaMemcpyHostToDevice, c->stream));
  MixedArgs g = mixed_args(c, m, precision);
  g.use_cond = 0;
  if (use_iter(c, m)) {  // one fused pass per iteration
    HPCCG_CUDA(cudaMemsetAsync(m->r2, 0, vec, c->stream));
    HPCCG_CUDA(cudaMemsetAsync(m->p2, 0, vec, c->stream));
    h0.passes = 1;
    HPCCG_CUDA(cudaMemcpyAsync(m->st, &h0, sizeof(MixedState), cudaMemcpyHostToDevice, c->stream));
    for (int rep = -1; rep < reps; ++rep) {
      if (rep == 0) HPCCG_CUDA(cudaEventRecord(c->ev0, c->stream));
      launch_iter(c, m, g, c->stream);
      HPCCG_CUDA(cudaGetLastError());
    }
    HPCCG_CUDA(cudaEventRecord(c->ev1, c->stream));
    HPCCG_CUDA(cudaEventSynchronize(c->ev1));
    float t = 0.f;
    HPCCG_CUDA(cudaEventElapsedTime(&t, c->ev0, c->ev1));
    ms[1] = t / (float)reps;
    // the FP64 refinement residual of an outer cycle (x and b as they stand)
    for (int rep = -1; rep < reps; ++rep) {
      if (rep == 0) HPCCG_CUDA(cudaEventRecord(c->ev0, c->stream));
      rc = launch_residual_f(c, m, g, c->stream, false);
      if (rc) return set_cuda_error((cudaError_t)rc, "residual", __FILE__, __LINE__);
    }
    HPCCG_CUDA(cudaEventRecord(c->ev1, c->stream));
    HPCCG_CUDA(cudaEventSynchronize(c->ev1));
    HPCCG_CUDA(cudaEventElapsedTime(&t, c->ev0, c->ev1));
    ms[0] = t / (float)reps;
    ms[2] = 0.f;
    return HPCCG_OK;
  }
  for (int which = 0; which < 3; ++which) {
    for (int rep = -1; rep < reps; ++rep) {
      if (rep == 0) HPCCG_CUDA(cudaEventRecord(c->ev0, c->stream));
      HPCCG_CUDA(cudaMemsetAsync(&m->st->inner_break, 0, sizeof(int), c->stream));
      if (which == 0) {
        k_mp_update_p<<<c->grid, kBlock, 0, c->stream>>>(g);
      } else if (which == 1 && use_tma(c, m)) {
        k_mp_spmv_dot_tma<<<tma_tile_grid(m->tile), kBlock, kTmaRingBytes, c->stream>>>(g, m->tile, m->pmap);
      } else if (which == 1) {
        dispatch_lp(uses_stencil(c), precision, m->rpt[precision], [&](auto strat, auto *vt) {
          using St = decltype(strat);
          using VT = std::remove_pointer_t<decltype(vt)>;
          k_mp_spmv_dot<St, VT><<<St::grid(g.pm, g.geom, c->grid), kBlock, 0, c->stream>>>(g);
          return 0;
        });
      } else {
        k_mp_update_r<<<c->grid, kBlock, 0, c->stream>>>(g);
      }
      HPCCG_CUDA(cudaGetLastError());
    }
    HPCCG_CUDA(cudaEventRecord(c->ev1, c->stream));
    HPCCG_CUDA(cudaEventSynchronize(c->ev1));
    float t = 0.f;
    HPCCG_CUDA(cudaEventElapsedTime(&t, c->ev0, c->ev1));
    ms[which] = t / (float)reps;
  }
  return HPCCG_OK;
}

// A flag of the context: allocates nothing (the next solve picks it up).
extern "C" int hpccg_gpu_set_mixed_fused(hpccg_ctx *c, int32_t on) {
  if (!c || (on != 0 && on != 1)) return HPCCG_ERR_INVALID_ARG;
  c->mixed_fused_off = on == 0;
  return HPCCG_OK;
}

extern "C" int hpccg_gpu_mixed_fused(hpccg_ctx *c, int32_t *fused) {
  if (!c || !fused) return HPCCG_ERR_INVALID_ARG;
  *fused = 0;
  if (!uses_stencil(c)) return HPCCG_OK;  // stored-matrix inner solves: three kernels (no values copied here)
  MixedRes *m = nullptr;
  const int rc = mixed_res(c, HPCCG_PREC_FP32, &m);
  if (rc) return rc;
  *fused = use_iter(c, m) ? 1 : 0;
  return HPCCG_OK;
}

extern "C" int hpccg_gpu_mixed_pass(hpccg_ctx *c, const float *d_r, const float *d_p, float *d_d, float *d_r_out,
                                    float *d_p_out, double alpha, double beta, int32_t first, double dots[4]) {
  if (!c || !d_r || !d_p || !d_d || !d_r_out || !d_p_out || !dots || (first != 0 && first != 1))
    return HPCCG_ERR_INVALID_ARG;
  MixedRes *m = nullptr;
  int rc = mixed_res(c, HPCCG_PREC_FP32, &m);
  if (rc) return rc;
  if (!uses_stencil(c) || !m->iter) return HPCCG_ERR_UNSUPPORTED;
  CUtensorMap pm, rm, dm;
  if (make_stencil_tmap(&pm, d_p, c->gx, c->gy, c->gz, kItPBoxY, kItBoxX) != HPCCG_OK ||
      make_stencil_tmap(&rm, d_r, c->gx, c->gy, c->gz, kItRBoxY, kItBoxX) != HPCCG_OK ||
      make_stencil_tmap(&dm, d_d, c->gx, c->gy, c->gz, kItTileY, kItTileX) != HPCCG_OK)
    return HPCCG_ERR_UNSUPPORTED;
  MixedState h0 = {};
  h0.alpha = alpha;
  h0.beta = beta;
  h0.passes = first ? 0 : 2;  // even: read the maps of buffer 0
  h0.max_inner = 1 << 30;
  h0.rr0 = 1.0;
  h0.scale = 1.0;  // the first pass divides r by it
  HPCCG_CUDA(cudaMemcpyAsync(m->st, &h0, sizeof(MixedState), cudaMemcpyHostToDevice, c->stream));
  MixedArgs g = mixed_args(c, m, HPCCG_PREC_FP32);
  g.use_cond = 0;
  g.d = d_d;
  const IterBufs b{{const_cast<float *>(d_r), d_r_out}, {const_cast<float *>(d_p), d_p_out}};
  k_mp_iter_tma<<<tma_tile_grid(m->itile), kItBlock, kItSmemBytes, c->stream>>>(g, m->itile, b, pm, pm, rm, rm, dm);
  HPCCG_CUDA(cudaGetLastError());
  MixedState hs;
  HPCCG_CUDA(cudaMemcpyAsync(&hs, m->st, sizeof(MixedState), cudaMemcpyDeviceToHost, c->stream));
  HPCCG_CUDA(cudaStreamSynchronize(c->stream));
  dots[0] = hs.pAp;
  dots[1] = hs.rAp;
  dots[2] = hs.ApAp;
  dots[3] = hs.rtrans;
  return hs.status ? hs.status : HPCCG_OK;
}
