// hpccg_batch.cu -- many independent HPCCG systems solved together.
//
// The systems are stacked block-diagonally in one column-major ELL (27 slots,
// global column indices); each system's rows start on a 512-row chunk
// boundary.  A schedule cuts every system into tiles of whole chunks; one
// persistent kernel per CG phase walks the tiles of all systems that are still
// active.  Every dot product is reduced per 512-row chunk in a fixed order
// (each lane's rows in order, then the fixed warp butterfly), and per system over its chunks in
// index order, so the result does not depend on the schedule: the autotuner
// may pick any tile size / grid and every iterate stays bit-identical.
//
// Solvers (all on the device, one CUDA graph with while nodes):
//   FP64: CG per system (same steps as MPI/src/numerics.F90:108-147, stopping
//         per system at ||r|| <= rel_tol ||b||), then an FP64 true residual.
//   FP32 / BF16: per-system FP64 iterative refinement around an inner CG in
//         FP32 vectors and FP32 / BF16 values (as hpccg_mixed.cu), with the
//         FP64 true residual as the stop test of every system.
// Batches built by hpccg_batch_create_generated may switch to matrix-free
// rows (hpccg_batch_set_spmv, HPCCG_SPMV_STENCIL): each row is formed from the
// system's own grid with the reference's term order (hpccg_stencil.cuh), so
// the FP64 iterates are bit-identical to the ELL rows'.
#include <stdlib.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "hpccg_internal.cuh"
#include "hpccg_rows_lp.cuh"
#include "hpccg_stencil.cuh"

namespace hpccg {

constexpr int kChunk = 512;  // rows per reduction chunk (16 per lane of one warp)

struct BatchSys {
  double bb, tol2, rtrans, pAp, alpha, beta, relres, scale, target, rr0;
  int k, active, status, outer, inner_k, inner_active, iters, converged;
};

struct BatchArgs {
  int nsys, ntiles;
  const int4 *tiles;        // (system, first row, end row, first chunk)
  const int *sys_chunk0;    // nsys+1 chunk offsets
  int npad;
  const int32_t *col;
  const double *val;
  const void *val_lp;
  double *x, *b, *r, *p, *Ap;
  float *r32, *p32, *Ap32, *d32;
  double *part;             // one partial per chunk
  unsigned *counter;
  BatchSys *sys;
  const int4 *dims;         // (nx, ny, nz, first row) per system: matrix-free rows; null = ELL
  const long long *walk;    // matrix-free rows: nsys+1 prefix of the column walks (columns x z chunks)
  double rel_tol, inner_rtol;
  int max_iter, max_outer, max_inner;
  cudaGraphConditionalHandle c_outer, c_inner;
  int use_cond;
};

// ---- per-row operations ------------------------------------------------------
__device__ __forceinline__ double row_fp64(const BatchArgs &g, int i, int sys, const double *x) {
  if (g.dims) {
    const int4 d = g.dims[sys];
    return stencil_row<double>(i - d.w, StencilGeom{d.x, d.y, d.z}, x + d.w);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const size_t o = (size_t)k * g.npad + i;
    s = __dadd_rn(s, __dmul_rn(__ldcs(g.val + o), __ldg(x + __ldcs(g.col + o))));
  }
  return s;
}

template <typename VT>
__device__ __forceinline__ float row_lp(const BatchArgs &g, int i, int sys, const float *x) {
  if (g.dims) {
    const int4 d = g.dims[sys];
    return stencil_row_box(i - d.w, StencilGeom{d.x, d.y, d.z}, x + d.w);  // FP32 inner solves: box sums
  }
  float s = 0.f;
  const VT *val = reinterpret_cast<const VT *>(g.val_lp);
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    const size_t o = (size_t)k * g.npad + i;
    float v[1];
    LpLoad<VT, 1>::vals(val, o, v);
    s = fmaf(v[0], __ldg(x + __ldcs(g.col + o)), s);
  }
  return s;
}

// ---- the phases ----------------------------------------------------------------
// Each phase: active(s) selects the systems it touches; value(i, s) reads and
// computes row i (no stores) and commit(i, s, v) stores it and returns the
// row's dot-product term, so a lane can issue the loads of kUnroll rows before
// any store (the vectors are not restrict-qualified and would otherwise be
// read one row at a time); finalize(s, total) runs once per active system in
// the last block; kCond names the loop condition it sets.
struct V2 {
  double a, b;
};
struct PhBnorm {  // bb = b.b
  static constexpr int kUnroll = 4;
  static constexpr bool kGather = false;
  static __device__ bool active(const BatchArgs &g, int s) { return true; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) { return {g.b[i], 0.0}; }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) { return __dmul_rn(v.a, v.a); }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.bb = t;
    y.tol2 = g.rel_tol * g.rel_tol * t;
    y.outer = 0;
    y.iters = 0;
    y.status = HPCCG_OK;
    y.converged = 0;
    y.active = 1;
  }
  static constexpr int kCond = -1;
};

struct PhInit64 {  // r = b - A x, p = r, rtrans = r.r
  static constexpr int kUnroll = 1;  // a row's 27 loads already overlap
  static constexpr bool kGather = true;
  static __device__ bool active(const BatchArgs &g, int s) { return true; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    return {__dsub_rn(g.b[i], row_fp64(g, i, s, g.x)), 0.0};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    g.r[i] = v.a;
    return __dmul_rn(v.a, v.a);
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.rtrans = t;
    y.k = 0;
    y.active = (t > y.tol2) && (g.max_iter > 0);
    y.converged = t <= y.tol2;  // false for a non-finite b, which then fails the final check
    y.relres = rel_residual(t, y.bb);
  }
  static constexpr int kCond = 1;  // outer (the CG loop)
};

struct PhSpmvDot64 {  // Ap = A p, alpha = rtrans / p.Ap
  static constexpr int kUnroll = 1;  // a row's 27 loads already overlap
  static constexpr bool kGather = true;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) { return {row_fp64(g, i, s, g.p), g.p[i]}; }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    g.Ap[i] = v.a;
    return __dmul_rn(v.b, v.a);
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.pAp = t;
    const double a = y.rtrans / t;
    if (!isfinite(a)) {
      y.status = HPCCG_ERR_BREAKDOWN;
      y.active = 0;
    } else {
      y.alpha = a;
    }
  }
  static constexpr int kCond = -1;
};

struct PhUpdate64 {  // x += alpha p, r -= alpha Ap, beta, per-system stop test
  static constexpr int kUnroll = 4;
  static constexpr bool kGather = false;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    const double a = g.sys[s].alpha;
    return {__dadd_rn(g.x[i], __dmul_rn(a, g.p[i])), __dadd_rn(g.r[i], __dmul_rn(-a, g.Ap[i]))};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    g.x[i] = v.a;
    g.r[i] = v.b;
    return __dmul_rn(v.b, v.b);
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.k += 1;
    y.iters = y.k;
    y.beta = t / y.rtrans;
    y.rtrans = t;
    if (!(t > y.tol2)) {
      y.active = 0;
      y.converged = 1;
    } else if (y.k >= g.max_iter || !isfinite(t)) {
      y.active = 0;
    }
  }
  static constexpr int kCond = 1;
};

struct PhResidual64 {  // final r = b - A x, relres (all systems)
  static constexpr int kUnroll = 1;  // a row's 27 loads already overlap
  static constexpr bool kGather = true;
  static __device__ bool active(const BatchArgs &g, int s) { return true; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    return {__dsub_rn(g.b[i], row_fp64(g, i, s, g.x)), 0.0};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) { return __dmul_rn(v.a, v.a); }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.relres = rel_residual(t, y.bb);
    y.converged = y.relres <= g.rel_tol;
  }
  static constexpr int kCond = -1;
};

// -- iterative refinement phases --
struct PhOuter64 {  // r64 = b - A x, relres, outer decision (systems still refining)
  static constexpr int kUnroll = 1;  // a row's 27 loads already overlap
  static constexpr bool kGather = true;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    return {__dsub_rn(g.b[i], row_fp64(g, i, s, g.x)), 0.0};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    g.r[i] = v.a;
    return __dmul_rn(v.a, v.a);
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.relres = rel_residual(t, y.bb);
    if (!isfinite(y.relres)) {
      y.status = HPCCG_ERR_BREAKDOWN;
      y.active = 0;
      return;
    }
    y.converged = y.relres <= g.rel_tol;
    y.active = !y.converged && y.outer < g.max_outer;
    if (y.active) {
      y.scale = sqrt(t);
      y.target = g.inner_rtol > 0.0 ? g.inner_rtol : fmax(1e-5, 0.5 * g.rel_tol / y.relres);
      y.outer += 1;
    }
  }
  static constexpr int kCond = 1;
};

struct PhStartInner {  // r32 = r64 / ||r64||, d = 0, rr0
  static constexpr int kUnroll = 4;
  static constexpr bool kGather = false;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    return {(double)(float)(g.r[i] / g.sys[s].scale), 0.0};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    const float ri = (float)v.a;
    g.r32[i] = ri;
    g.d32[i] = 0.f;
    return (double)ri * ri;
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.rtrans = t;
    y.rr0 = t;
    y.inner_k = 0;
    y.inner_active = t > 0.0 && g.max_inner > 0;
  }
  static constexpr int kCond = 2;  // inner
};

template <typename VT>
struct PhSpmvDotLp {
  static constexpr int kUnroll = 1;  // a row's 27 loads already overlap
  static constexpr bool kGather = true;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].inner_active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    return {(double)row_lp<VT>(g, i, s, g.p32), (double)g.p32[i]};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    const float ai = (float)v.a;
    g.Ap32[i] = ai;
    return v.b * ai;
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    const double a = y.rtrans / t;
    if (!(t > 0.0) || !isfinite(a)) {
      y.inner_active = 0;
      y.alpha = 0.0;
    } else {
      y.alpha = a;
    }
  }
  static constexpr int kCond = -1;
};

struct PhUpdateLp {  // d += alpha p, r -= alpha Ap, inner stop test
  static constexpr int kUnroll = 4;
  static constexpr bool kGather = false;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].inner_active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) {
    const float a = (float)g.sys[s].alpha;
    return {(double)fmaf(a, g.p32[i], g.d32[i]), (double)fmaf(-a, g.Ap32[i], g.r32[i])};
  }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) {
    const float ri = (float)v.b;
    g.d32[i] = (float)v.a;
    g.r32[i] = ri;
    return (double)ri * ri;
  }
  static __device__ void finalize(const BatchArgs &g, int s, double t) {
    BatchSys &y = g.sys[s];
    y.inner_k += 1;
    y.iters += 1;
    y.beta = t / y.rtrans;
    y.rtrans = t;
    y.inner_active = isfinite(t) && t > y.target * y.target * y.rr0 && y.inner_k < g.max_inner;
  }
  static constexpr int kCond = 2;
};

// Matrix-free batches form A p by column walks (k_batch_walk64 / 32 below) and
// then reduce p.Ap here, in the same chunk order as PhSpmvDot64 / PhSpmvDotLp.
struct PhDot64 {  // alpha = rtrans / p.Ap
  static constexpr int kUnroll = 4;
  static constexpr bool kGather = false;
  static __device__ bool active(const BatchArgs &g, int s) { return PhSpmvDot64::active(g, s); }
  static __device__ V2 value(const BatchArgs &g, int i, int s) { return {g.Ap[i], g.p[i]}; }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) { return __dmul_rn(v.b, v.a); }
  static __device__ void finalize(const BatchArgs &g, int s, double t) { PhSpmvDot64::finalize(g, s, t); }
  static constexpr int kCond = -1;
};
struct PhDotLp {
  static constexpr int kUnroll = 4;
  static constexpr bool kGather = false;
  static __device__ bool active(const BatchArgs &g, int s) { return g.sys[s].inner_active; }
  static __device__ V2 value(const BatchArgs &g, int i, int s) { return {(double)g.Ap32[i], (double)g.p32[i]}; }
  static __device__ double commit(const BatchArgs &g, int i, int s, const V2 &v) { return v.b * (float)v.a; }
  static __device__ void finalize(const BatchArgs &g, int s, double t) { PhSpmvDotLp<float>::finalize(g, s, t); }
  static constexpr int kCond = -1;
};

// ---- column walks of matrix-free batches -------------------------------------------
constexpr int kWalkZc = 32;  // z planes per walk

// The walk of work item t: system, column and z range (prefix g.walk).
struct WalkItem {
  int s, c, z0, z1;
  int4 d;
};
__device__ __forceinline__ bool walk_item(const BatchArgs &g, long long t, WalkItem &w) {
  if (t >= g.walk[g.nsys]) return false;
  int lo = 0, hi = g.nsys;  // g.walk[lo] <= t < g.walk[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (g.walk[mid] <= t) lo = mid;
    else hi = mid;
  }
  w.s = lo;
  w.d = g.dims[lo];
  const int plane = w.d.x * w.d.y;
  const long long local = t - g.walk[lo];
  const int q = (int)(local / plane);
  w.c = (int)(local - (long long)q * plane);
  w.z0 = q * kWalkZc;
  w.z1 = min(w.d.z, w.z0 + kWalkZc);
  return true;
}

struct WalkStore {  // y[i] = row sum (stencil_column's epilogue)
  double *y;
  __device__ __forceinline__ double operator()(int i, double s, double) const {
    y[i] = s;
    return 0.0;
  }
};

// Ap = A p of the active systems (FP64, reference term order: the rows equal
// the ones PhSpmvDot64 forms, bit for bit).
__global__ void __launch_bounds__(256, 4) k_batch_walk64(BatchArgs g) {
  WalkItem w;
  const bool have = walk_item(g, blockIdx.x * 256LL + threadIdx.x, w) && g.sys[w.s].active;
  if (!have) return;
  const StencilGeom geom{w.d.x, w.d.y, w.d.z};
  const PlaneMap m{w.d.x * w.d.y, kWalkZc, 0, 1};
  const PlaneSpan sp{w.c, w.z0, w.z1};
  const int iy = w.c / w.d.x, ix = w.c - iy * w.d.x;
  const unsigned mask = stencil_mask(geom, ix, iy);
  WalkStore epi{g.Ap + w.d.w};
  if (__all_sync(__activemask(), mask == 0x1FFu))
    stencil_column_interior<double>(sp, geom, m, g.p + w.d.w + w.c, epi);
  else
    stencil_column<double>(sp, geom, m, mask, g.p + w.d.w + w.c, epi);
}

// The same for the FP32 inner solves, rows as 28 x - (plane box sums), the
// form of stencil_row_box.
__device__ __forceinline__ float walk_box32(const float *__restrict__ x, int nx, unsigned mask) {
  float ln[3];
#pragma unroll
  for (int sy = 0; sy < 3; ++sy) {
    const float *r = x + (sy - 1) * nx;
    const float l = ((mask >> (3 * sy)) & 1u) ? __ldg(r - 1) : 0.f;
    const float c = ((mask >> (3 * sy + 1)) & 1u) ? __ldg(r) : 0.f;
    const float rr = ((mask >> (3 * sy + 2)) & 1u) ? __ldg(r + 1) : 0.f;
    ln[sy] = (l + c) + rr;
  }
  return (ln[0] + ln[1]) + ln[2];
}
__global__ void __launch_bounds__(256, 4) k_batch_walk32(BatchArgs g) {
  WalkItem w;
  const bool have = walk_item(g, blockIdx.x * 256LL + threadIdx.x, w) && g.sys[w.s].inner_active;
  if (!have) return;
  const int plane = w.d.x * w.d.y;
  const int iy = w.c / w.d.x, ix = w.c - iy * w.d.x;
  const unsigned mask = stencil_mask(StencilGeom{w.d.x, w.d.y, w.d.z}, ix, iy);
  const float *pc = g.p32 + w.d.w + w.c;
  float *y = g.Ap32 + w.d.w + w.c;
  float bm = w.z0 > 0 ? walk_box32(pc + (int64_t)(w.z0 - 1) * plane, w.d.x, mask) : 0.f;
  float b0 = walk_box32(pc + (int64_t)w.z0 * plane, w.d.x, mask);
  for (int z = w.z0; z < w.z1; ++z) {
    const float bp = z + 1 < w.d.z ? walk_box32(pc + (int64_t)(z + 1) * plane, w.d.x, mask) : 0.f;
    y[(int64_t)z * plane] = fmaf(28.f, __ldg(pc + (int64_t)z * plane), -((bm + b0) + bp));
    bm = b0;
    b0 = bp;
  }
}

// ---- the persistent phase kernel --------------------------------------------------
__device__ __forceinline__ void set_cond(const BatchArgs &g, int which, int v) {
  if (!g.use_cond || which < 0) return;
  cudaGraphSetConditional(which == 1 ? g.c_outer : g.c_inner, (unsigned)v);
}

// Each warp takes whole tiles (tile t goes to warp t mod the grid's warps).
// A chunk's partial: lane l sums rows r0 + l + 32k, k = 0..15, in k order,
// then the fixed warp butterfly; so it depends on neither the schedule nor
// the warp that forms it.
// Stored-matrix rows of the SpMV phases (gathers through the column indices)
// want more rows in flight: a block takes whole tiles, warp w reads rows
// r0 + l + 32k for k = 2w, 2w+1, and warp 0 sums each lane's 16 terms in k
// order before the butterfly, so the partial equals the one-warp form's bit
// for bit (a row past the tile adds +0.0, which never changes such a sum).
template <class Ph>
__device__ __forceinline__ void phase_block_tiles(const BatchArgs &g, double (*sv)[32]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x) {
    const int4 tile = g.tiles[t];
    const int s = tile.x;
    if (!Ph::active(g, s)) continue;  // uniform over the block
    const int nch = (tile.z - tile.y + kChunk - 1) / kChunk;
    for (int c = 0; c < nch; ++c) {
      const int r0 = tile.y + c * kChunk, rend = min(tile.z, r0 + kChunk);
      V2 val[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = r0 + (2 * w + u) * 32 + lane;
        if (i < rend) val[u] = Ph::value(g, i, s);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int i = r0 + (2 * w + u) * 32 + lane;
        sv[2 * w + u][lane] = i < rend ? Ph::commit(g, i, s, val[u]) : 0.0;
      }
      __syncthreads();
      if (w == 0) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kChunk / 32; ++k) v = __dadd_rn(v, sv[k][lane]);
        v = warp_sum(v);
        if (lane == 0) {
          g.part[tile.w + c] = v;
          __threadfence();
        }
      }
      __syncthreads();
    }
  }
}

template <class Ph>
__global__ void __launch_bounds__(256, 4) k_batch_phase(BatchArgs g) {
  __shared__ bool s_last;
  __shared__ double sv[kChunk / 32][32];
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * 8;
  if (Ph::kGather && !g.dims) {
    phase_block_tiles<Ph>(g, sv);
  } else
  for (int t = blockIdx.x * 8 + (threadIdx.x >> 5); t < g.ntiles; t += nw) {
    const int4 tile = g.tiles[t];
    const int s = tile.x;
    if (!Ph::active(g, s)) continue;  // uniform over the warp
    const int nch = (tile.z - tile.y + kChunk - 1) / kChunk;
    for (int c = 0; c < nch; ++c) {
      const int r0 = tile.y + c * kChunk, rend = min(tile.z, r0 + kChunk);
      double v = 0.0;
      for (int k0 = 0; k0 < kChunk / 32; k0 += Ph::kUnroll) {
        V2 val[Ph::kUnroll];
#pragma unroll
        for (int u = 0; u < Ph::kUnroll; ++u) {
          const int i = r0 + (k0 + u) * 32 + lane;
          if (i < rend) val[u] = Ph::value(g, i, s);
        }
#pragma unroll
        for (int u = 0; u < Ph::kUnroll; ++u) {
          const int i = r0 + (k0 + u) * 32 + lane;
          if (i < rend) v = __dadd_rn(v, Ph::commit(g, i, s, val[u]));
        }
      }
      v = warp_sum(v);
      if (lane == 0) {
        g.part[tile.w + c] = v;
        __threadfence();
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(g.counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // one warp per system: lanes stride the system's chunks, fixed butterfly
  const int warp = threadIdx.x >> 5;
  for (int s = warp; s < g.nsys; s += 8) {
    if (!Ph::active(g, s)) continue;
    double v = 0.0;
    for (int c = g.sys_chunk0[s] + lane; c < g.sys_chunk0[s + 1]; c += 32)
      v = __dadd_rn(v, ((volatile double *)g.part)[c]);
    v = warp_sum(v);
    if (lane == 0) Ph::finalize(g, s, v);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *g.counter = 0u;
    if (Ph::kCond >= 0) {
      int any = 0;
      for (int s = 0; s < g.nsys; ++s) {
        const volatile BatchSys &y = g.sys[s];
        any |= Ph::kCond == 2 ? y.inner_active : y.active;
      }
      set_cond(g, Ph::kCond, any);
    }
  }
}

// Element-wise phases without a reduction, persistent over the same tiles
// (one warp per tile, 32 consecutive rows per step; each lane reads four rows
// before it stores any, as in the phases above).
template <class F>
__device__ __forceinline__ void batch_rows4(int lo, int hi, F &&f) {
  const int lane = threadIdx.x & 31;
  for (int i0 = lo + lane; i0 < hi; i0 += 128) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i0 + 32 * u < hi) v[u] = f.value(i0 + 32 * u);
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i0 + 32 * u < hi) f.commit(i0 + 32 * u, v[u]);
  }
}

__global__ void __launch_bounds__(256) k_batch_p64(BatchArgs g) {
  const int nw = gridDim.x * 8;
  for (int t = blockIdx.x * 8 + (threadIdx.x >> 5); t < g.ntiles; t += nw) {
    const int4 tile = g.tiles[t];
    const BatchSys &y = g.sys[tile.x];
    if (!y.active) continue;
    struct {
      const BatchArgs &g;
      bool first;
      double beta;
      __device__ double value(int i) const { return first ? g.r[i] : __dadd_rn(g.r[i], __dmul_rn(beta, g.p[i])); }
      __device__ void commit(int i, double v) const { g.p[i] = v; }
    } f{g, y.k == 0, y.beta};
    batch_rows4(tile.y, tile.z, f);
  }
}

__global__ void __launch_bounds__(256) k_batch_p32(BatchArgs g) {
  const int nw = gridDim.x * 8;
  for (int t = blockIdx.x * 8 + (threadIdx.x >> 5); t < g.ntiles; t += nw) {
    const int4 tile = g.tiles[t];
    const BatchSys &y = g.sys[tile.x];
    if (!y.inner_active) continue;
    struct {
      const BatchArgs &g;
      bool first;
      float beta;
      __device__ double value(int i) const { return first ? g.r32[i] : fmaf(beta, g.p32[i], g.r32[i]); }
      __device__ void commit(int i, double v) const { g.p32[i] = (float)v; }
    } f{g, y.inner_k == 0, (float)y.beta};
    batch_rows4(tile.y, tile.z, f);
  }
}

__global__ void __launch_bounds__(256) k_batch_end_inner(BatchArgs g) {
  const int nw = gridDim.x * 8;
  for (int t = blockIdx.x * 8 + (threadIdx.x >> 5); t < g.ntiles; t += nw) {
    const int4 tile = g.tiles[t];
    const BatchSys &y = g.sys[tile.x];
    if (!y.active) continue;
    struct {
      const BatchArgs &g;
      double scale;
      __device__ double value(int i) const { return fma(scale, (double)g.d32[i], g.x[i]); }
      __device__ void commit(int i, double v) const { g.x[i] = v; }
    } f{g, y.scale};
    batch_rows4(tile.y, tile.z, f);
  }
}

// Plain FP64 y = A x over all systems (tests, b = A x*).
__global__ void k_batch_spmv(BatchArgs g, const double *x, double *y) {
  for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x) {
    const int4 tile = g.tiles[t];
    for (int i = tile.y + threadIdx.x; i < tile.z; i += 256) y[i] = row_fp64(g, i, tile.x, x);
  }
}

// generate_matrix(nx,ny,nz) rows written into the stacked ELL at row offset `off`.
__global__ void k_batch_generate(int nx, int ny, int nz, int off, int npad, int32_t *col, double *val) {
  const int n = nx * ny * nz;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int ix = row % nx + 1, iy = (row / nx) % ny + 1, iz = row / (nx * ny) + 1;
    int k = 0;
    for (int sz = (iz > 1 ? -1 : 0); sz <= (iz < nz ? 1 : 0); ++sz)
      for (int sy = (iy > 1 ? -1 : 0); sy <= (iy < ny ? 1 : 0); ++sy)
        for (int sx = (ix > 1 ? -1 : 0); sx <= (ix < nx ? 1 : 0); ++sx) {
          const size_t o = (size_t)k * npad + off + row;
          col[o] = off + row + sz * nx * ny + sy * nx + sx;
          val[o] = (sz == 0 && sy == 0 && sx == 0) ? 27.0 : -1.0;
          ++k;
        }
    for (; k < 27; ++k) {
      const size_t o = (size_t)k * npad + off + row;
      col[o] = off + row;
      val[o] = 0.0;
    }
  }
}

// 1-based CSR rows of one system into the stacked ELL at row offset `off`.
__global__ void k_batch_from_csr(int n, const int32_t *rowindex, const int32_t *colindex, const double *values,
                                 int off, int npad, int32_t *col, double *val, int *bad) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    const int a = rowindex[row] - 1, e = rowindex[row + 1] - 1;
    if (e < a || e - a > 27) {
      atomicOr(bad, 1);
      continue;
    }
    for (int k = 0; k < 27; ++k) {
      const size_t o = (size_t)k * npad + off + row;
      if (k < e - a) {
        const int c = colindex[a + k];
        if (c < 1 || c > n) atomicOr(bad, 2);
        col[o] = off + (c >= 1 && c <= n ? c - 1 : row);
        val[o] = values[a + k];
      } else {
        col[o] = off + row;
        val[o] = 0.0;
      }
    }
  }
}

__global__ void k_batch_pad(int npad, int32_t *col, double *val, const int *is_row) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npad; i += gridDim.x * blockDim.x)
    if (!is_row[i])
      for (int k = 0; k < 27; ++k) {
        col[(size_t)k * npad + i] = i;
        val[(size_t)k * npad + i] = 0.0;
      }
}

}  // namespace hpccg

using namespace hpccg;

struct hpccg_batch {
  int device = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int nsys = 0;
  int npad = 0;
  std::vector<int> n, off, chunk0;  // per system rows, row offset, first chunk (host copies)
  int nchunks = 0;
  int32_t *col = nullptr;
  double *val = nullptr;
  float *val32 = nullptr;
  __nv_bfloat16 *val16 = nullptr;
  double *x = nullptr, *b = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr;
  float *r32 = nullptr, *p32 = nullptr, *Ap32 = nullptr, *d32 = nullptr;
  double *part = nullptr;
  unsigned *counter = nullptr;
  BatchSys *sys = nullptr;
  int *d_sys_chunk0 = nullptr;
  int4 *d_tiles = nullptr;
  int4 *d_dims = nullptr;  // generated batches: (nx, ny, nz, first row) per system
  long long *d_walk = nullptr;  // and the prefix of their column walks (nsys+1)
  long long walk_total = 0;
  int spmv_kind = HPCCG_SPMV_ELL;
  int ntiles = 0;
  int tile_chunks = 0, blocks_per_sm = 0;  // schedule; 0 = not tuned yet
  bool tuned = false;
  cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
  int exec_tile[3] = {0, 0, 0}, exec_bps[3] = {0, 0, 0}, exec_maxit[3] = {-1, -1, -1}, exec_kind[3] = {0, 0, 0};
  double exec_tol[3] = {-1.0, -1.0, -1.0};
  float last_ms = 0.f;
};

static void batch_free(hpccg_batch *B) {
  for (auto &e : B->exec)
    if (e) cudaGraphExecDestroy(e);
  void *bufs[] = {B->col, B->val, B->val32, B->val16, B->x, B->b, B->r, B->p, B->Ap, B->r32, B->p32,
                  B->Ap32, B->d32, B->part, B->counter, B->sys, B->d_sys_chunk0, B->d_tiles, B->d_dims, B->d_walk};
  for (void *q : bufs)
    if (q) cudaFree(q);
  if (B->ev0) cudaEventDestroy(B->ev0);
  if (B->ev1) cudaEventDestroy(B->ev1);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
}

static int build_tiles(hpccg_batch *B, int tile_chunks) {
  std::vector<int4> tiles;
  for (int s = 0; s < B->nsys; ++s) {
    const int rows_per_tile = tile_chunks * kChunk;
    for (int r0 = 0; r0 < B->n[s]; r0 += rows_per_tile) {
      const int r1 = std::min(B->n[s], r0 + rows_per_tile);
      tiles.push_back(make_int4(s, B->off[s] + r0, B->off[s] + r1, B->chunk0[s] + r0 / kChunk));
    }
  }
  if (B->d_tiles) cudaFree(B->d_tiles);
  B->d_tiles = nullptr;
  HPCCG_CUDA(cudaMalloc(&B->d_tiles, sizeof(int4) * tiles.size()));
  HPCCG_CUDA(cudaMemcpyAsync(B->d_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, B->stream));
  HPCCG_CUDA(cudaStreamSynchronize(B->stream));
  B->ntiles = (int)tiles.size();
  B->tile_chunks = tile_chunks;
  return HPCCG_OK;
}

// Lays out the systems (rows on 512-row boundaries) and allocates everything.
static int batch_alloc(hpccg_batch *B, int nsys, const int64_t *rows) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HPCCG_ERR_NO_DEVICE;
  HPCCG_CUDA(cudaGetDevice(&B->device));
  HPCCG_CUDA(cudaDeviceGetAttribute(&B->num_sms, cudaDevAttrMultiProcessorCount, B->device));
  HPCCG_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
  HPCCG_CUDA(cudaEventCreate(&B->ev0));
  HPCCG_CUDA(cudaEventCreate(&B->ev1));
  B->nsys = nsys;
  int64_t off = 0, chunks = 0;
  for (int s = 0; s < nsys; ++s) {
    B->n.push_back((int)rows[s]);
    B->off.push_back((int)off);
    B->chunk0.push_back((int)chunks);
    const int64_t c = (rows[s] + kChunk - 1) / kChunk;
    chunks += c;
    off += c * kChunk;
  }
  B->chunk0.push_back((int)chunks);
  if (off * 27 > INT32_MAX) return HPCCG_ERR_INVALID_ARG;
  B->npad = (int)off;
  B->nchunks = (int)chunks;
  const size_t slots = (size_t)27 * B->npad;
  HPCCG_CUDA(cudaMalloc(&B->col, sizeof(int32_t) * slots));
  HPCCG_CUDA(cudaMalloc(&B->val, sizeof(double) * slots));
  const size_t v64 = sizeof(double) * B->npad, v32 = sizeof(float) * B->npad;
  double **d64[] = {&B->x, &B->b, &B->r, &B->p, &B->Ap};
  for (double **q : d64) {
    HPCCG_CUDA(cudaMalloc(q, v64));
    HPCCG_CUDA(cudaMemsetAsync(*q, 0, v64, B->stream));
  }
  float **d32[] = {&B->r32, &B->p32, &B->Ap32, &B->d32};
  for (float **q : d32) {
    HPCCG_CUDA(cudaMalloc(q, v32));
    HPCCG_CUDA(cudaMemsetAsync(*q, 0, v32, B->stream));
  }
  HPCCG_CUDA(cudaMalloc(&B->part, sizeof(double) * std::max(1, B->nchunks)));
  HPCCG_CUDA(cudaMalloc(&B->counter, sizeof(unsigned) * 4));
  HPCCG_CUDA(cudaMemsetAsync(B->counter, 0, sizeof(unsigned) * 4, B->stream));
  HPCCG_CUDA(cudaMalloc(&B->sys, sizeof(BatchSys) * nsys));
  HPCCG_CUDA(cudaMemsetAsync(B->sys, 0, sizeof(BatchSys) * nsys, B->stream));
  HPCCG_CUDA(cudaMalloc(&B->d_sys_chunk0, sizeof(int) * (nsys + 1)));
  HPCCG_CUDA(cudaMemcpyAsync(B->d_sys_chunk0, B->chunk0.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice,
                             B->stream));
  HPCCG_CUDA(cudaStreamSynchronize(B->stream));
  B->blocks_per_sm = 4;
  return build_tiles(B, 4);
}

// Marks padding rows (between systems) so they multiply as exact zeros.
static int batch_pad_rows(hpccg_batch *B) {
  std::vector<int> is_row(B->npad, 0);
  for (int s = 0; s < B->nsys; ++s)
    for (int i = 0; i < B->n[s]; ++i) is_row[B->off[s] + i] = 1;
  int *d = nullptr;
  HPCCG_CUDA(cudaMalloc(&d, sizeof(int) * B->npad));
  cudaMemcpyAsync(d, is_row.data(), sizeof(int) * B->npad, cudaMemcpyHostToDevice, B->stream);
  k_batch_pad<<<B->num_sms * 8, 256, 0, B->stream>>>(B->npad, B->col, B->val, d);
  const cudaError_t e = cudaStreamSynchronize(B->stream);
  cudaFree(d);
  HPCCG_CUDA(e);
  return HPCCG_OK;
}

extern "C" int hpccg_batch_create_generated(int32_t nsys, const int32_t *sizes, hpccg_batch **out) {
  if (!out || nsys < 1 || !sizes) return HPCCG_ERR_INVALID_ARG;
  std::vector<int64_t> rows(nsys);
  for (int s = 0; s < nsys; ++s) {
    if (sizes[3 * s] < 1 || sizes[3 * s + 1] < 1 || sizes[3 * s + 2] < 1) return HPCCG_ERR_INVALID_ARG;
    rows[s] = (int64_t)sizes[3 * s] * sizes[3 * s + 1] * sizes[3 * s + 2];
    if (rows[s] * 27 > INT32_MAX) return HPCCG_ERR_INVALID_ARG;
  }
  *out = nullptr;
  hpccg_batch *B = new hpccg_batch();
  int rc = batch_alloc(B, nsys, rows.data());
  if (rc) {
    batch_free(B);
    return rc;
  }
  for (int s = 0; s < nsys; ++s)
    k_batch_generate<<<B->num_sms * 8, 256, 0, B->stream>>>(sizes[3 * s], sizes[3 * s + 1], sizes[3 * s + 2],
                                                             B->off[s], B->npad, B->col, B->val);
  {
    std::vector<int4> dims(nsys);
    std::vector<long long> walk(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) {
      dims[s] = make_int4(sizes[3 * s], sizes[3 * s + 1], sizes[3 * s + 2], B->off[s]);
      const long long chunks = (sizes[3 * s + 2] + kWalkZc - 1) / kWalkZc;
      walk[s + 1] = walk[s] + (long long)sizes[3 * s] * sizes[3 * s + 1] * chunks;
    }
    B->walk_total = walk[nsys];
    cudaError_t e = cudaMalloc(&B->d_dims, sizeof(int4) * nsys);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(B->d_dims, dims.data(), sizeof(int4) * nsys, cudaMemcpyHostToDevice, B->stream);
    if (e == cudaSuccess) e = cudaMalloc(&B->d_walk, sizeof(long long) * (nsys + 1));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(B->d_walk, walk.data(), sizeof(long long) * (nsys + 1), cudaMemcpyHostToDevice, B->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    if (e != cudaSuccess) {
      batch_free(B);
      return set_cuda_error(e, "batch dims", __FILE__, __LINE__);
    }
  }
  if ((rc = batch_pad_rows(B))) {
    batch_free(B);
    return rc;
  }
  *out = B;
  return HPCCG_OK;
}

extern "C" int hpccg_batch_create(int32_t nsys, const int32_t *nrows, const int32_t *const *rowindex,
                                  const int32_t *const *colindex, const double *const *values,
                                  hpccg_batch **out) {
  if (!out || nsys < 1 || !nrows || !rowindex || !colindex || !values) return HPCCG_ERR_INVALID_ARG;
  std::vector<int64_t> rows(nsys);
  for (int s = 0; s < nsys; ++s) {
    if (nrows[s] < 1 || !rowindex[s]) return HPCCG_ERR_INVALID_ARG;
    rows[s] = nrows[s];
  }
  *out = nullptr;
  hpccg_batch *B = new hpccg_batch();
  int rc = batch_alloc(B, nsys, rows.data());
  int *d_bad = nullptr;
  int bad = 0;
  if (!rc && cudaMalloc(&d_bad, sizeof(int)) != cudaSuccess) rc = HPCCG_ERR_OOM;
  if (!rc) cudaMemsetAsync(d_bad, 0, sizeof(int), B->stream);
  for (int s = 0; s < nsys && !rc; ++s) {
    const int n = nrows[s];
    const int64_t nnz = (int64_t)rowindex[s][n] - 1;
    if (nnz < 0 || nnz > 27 * (int64_t)n || (nnz > 0 && (!colindex[s] || !values[s]))) {
      rc = HPCCG_ERR_INVALID_ARG;
      break;
    }
    int32_t *dr = nullptr, *dc = nullptr;
    double *dv = nullptr;
    if (cudaMalloc(&dr, sizeof(int32_t) * (n + 1)) != cudaSuccess ||
        cudaMalloc(&dc, sizeof(int32_t) * std::max<int64_t>(nnz, 1)) != cudaSuccess ||
        cudaMalloc(&dv, sizeof(double) * std::max<int64_t>(nnz, 1)) != cudaSuccess) {
      rc = HPCCG_ERR_OOM;
    } else {
      // copies and kernel on the batch stream, so the kernel sees finished copies
      cudaMemcpyAsync(dr, rowindex[s], sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice, B->stream);
      if (nnz > 0) {
        cudaMemcpyAsync(dc, colindex[s], sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, B->stream);
        cudaMemcpyAsync(dv, values[s], sizeof(double) * nnz, cudaMemcpyHostToDevice, B->stream);
      }
      k_batch_from_csr<<<B->num_sms * 8, 256, 0, B->stream>>>(n, dr, dc, dv, B->off[s], B->npad, B->col,
                                                               B->val, d_bad);
      if (cudaStreamSynchronize(B->stream) != cudaSuccess) rc = set_cuda_error(cudaGetLastError(), "batch csr", __FILE__, __LINE__);
    }
    if (dr) cudaFree(dr);
    if (dc) cudaFree(dc);
    if (dv) cudaFree(dv);
  }
  if (!rc) {
    cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, B->stream);
    cudaStreamSynchronize(B->stream);
    if (bad) rc = HPCCG_ERR_INVALID_ARG;
  }
  if (d_bad) cudaFree(d_bad);
  if (!rc) rc = batch_pad_rows(B);
  if (rc) {
    batch_free(B);
    return rc;
  }
  *out = B;
  return HPCCG_OK;
}

extern "C" void hpccg_batch_destroy(hpccg_batch *B) {
  if (B) batch_free(B);
}

extern "C" int hpccg_batch_info(const hpccg_batch *B, int32_t *nsys, int64_t *stacked_rows,
                                int64_t *row_offsets) {
  if (!B) return HPCCG_ERR_INVALID_ARG;
  if (nsys) *nsys = B->nsys;
  if (stacked_rows) *stacked_rows = B->npad;
  if (row_offsets)
    for (int s = 0; s < B->nsys; ++s) {
      row_offsets[2 * s] = B->off[s];
      row_offsets[2 * s + 1] = B->n[s];
    }
  return HPCCG_OK;
}

static BatchArgs batch_args(hpccg_batch *B, int precision) {
  BatchArgs g{};
  g.nsys = B->nsys;
  g.ntiles = B->ntiles;
  g.tiles = B->d_tiles;
  g.sys_chunk0 = B->d_sys_chunk0;
  g.npad = B->npad;
  g.col = B->col;
  g.val = B->val;
  g.val_lp = precision == HPCCG_PREC_BF16 ? (const void *)B->val16 : (const void *)B->val32;
  g.x = B->x;
  g.b = B->b;
  g.r = B->r;
  g.p = B->p;
  g.Ap = B->Ap;
  g.r32 = B->r32;
  g.p32 = B->p32;
  g.Ap32 = B->Ap32;
  g.d32 = B->d32;
  g.part = B->part;
  g.counter = B->counter;
  g.sys = B->sys;
  g.dims = B->spmv_kind == HPCCG_SPMV_STENCIL ? B->d_dims : nullptr;
  g.walk = B->d_walk;
  return g;
}

static int grid_of(const hpccg_batch *B) { return B->num_sms * B->blocks_per_sm; }

template <class Ph>
static cudaError_t phase(hpccg_batch *B, const BatchArgs &g, cudaStream_t s) {
  k_batch_phase<Ph><<<grid_of(B), 256, 0, s>>>(g);
  return cudaGetLastError();
}

static int walk_grid(const hpccg_batch *B) { return (int)((B->walk_total + 255) / 256); }

// Ap = A p and alpha: one phase on the stored matrix, a column walk and a dot
// phase on matrix-free rows.
static cudaError_t launch_spmv_dot64(hpccg_batch *B, const BatchArgs &g, cudaStream_t s) {
  if (g.dims && g.walk && B->walk_total > 0) {
    k_batch_walk64<<<walk_grid(B), 256, 0, s>>>(g);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? phase<PhDot64>(B, g, s) : e;
  }
  return phase<PhSpmvDot64>(B, g, s);
}

static cudaError_t launch_cg64_body(hpccg_batch *B, const BatchArgs &g, cudaStream_t s) {
  k_batch_p64<<<grid_of(B), 256, 0, s>>>(g);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_spmv_dot64(B, g, s);
  if (e == cudaSuccess) e = phase<PhUpdate64>(B, g, s);
  return e;
}

template <typename VT>
static cudaError_t launch_inner_body(hpccg_batch *B, const BatchArgs &g, cudaStream_t s) {
  k_batch_p32<<<grid_of(B), 256, 0, s>>>(g);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    if (g.dims && g.walk && B->walk_total > 0) {
      k_batch_walk32<<<walk_grid(B), 256, 0, s>>>(g);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = phase<PhDotLp>(B, g, s);
    } else {
      e = phase<PhSpmvDotLp<VT>>(B, g, s);
    }
  }
  if (e == cudaSuccess) e = phase<PhUpdateLp>(B, g, s);
  return e;
}

template <typename VT>
static cudaError_t launch_outer_body(hpccg_batch *B, const BatchArgs &g, cudaStream_t s,
                                     cudaGraph_t og, bool graph) {
  cudaError_t e = phase<PhStartInner>(B, g, s);
  if (e != cudaSuccess) return e;
  if (graph) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = g.c_inner;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&node, cg, deps, nd, &cp);
    }
    cudaStream_t is = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&is, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(is, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const cudaError_t e1 = launch_inner_body<VT>(B, g, is);
        const cudaError_t e2 = cudaStreamEndCapture(is, &body);
        e = e1 != cudaSuccess ? e1 : e2;
      }
      cudaStreamDestroy(is);
    }
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
  } else {
    for (;;) {
      int any = 0;
      std::vector<BatchSys> hs(B->nsys);
      e = cudaMemcpyAsync(hs.data(), B->sys, sizeof(BatchSys) * B->nsys, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return e;
      for (auto &y : hs) any |= y.inner_active;
      if (!any) break;
      if ((e = launch_inner_body<VT>(B, g, s)) != cudaSuccess) return e;
    }
  }
  if (e != cudaSuccess) return e;
  k_batch_end_inner<<<grid_of(B), 256, 0, s>>>(g);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = phase<PhOuter64>(B, g, s);
  return e;
}

constexpr int kBatchMaxOuter = 30;  // refinement cycles per system (mixed precision)

// Captures the solver for one precision as a graph (or runs it eagerly).  The
// solve parameters travel in the kernel arguments, so a graph is rebuilt when
// they or the schedule change.
static int run_batch(hpccg_batch *B, int precision, bool eager, double rel_tol, int max_iter) {
  cudaStream_t s = B->stream;
  BatchArgs g = batch_args(B, precision);
  g.rel_tol = rel_tol;
  g.max_iter = max_iter;
  g.max_inner = max_iter;
  g.max_outer = kBatchMaxOuter;
  g.inner_rtol = 0.0;
  if (eager) {
    g.use_cond = 0;
    auto any_active = [&](int &any) -> cudaError_t {
      std::vector<BatchSys> hs(B->nsys);
      cudaError_t e = cudaMemcpyAsync(hs.data(), B->sys, sizeof(BatchSys) * B->nsys, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      any = 0;
      for (auto &y : hs) any |= y.active;
      return e;
    };
    HPCCG_CUDA(phase<PhBnorm>(B, g, s));
    if (precision == HPCCG_PREC_FP64) {
      HPCCG_CUDA(phase<PhInit64>(B, g, s));
      for (;;) {
        int any = 0;
        HPCCG_CUDA(any_active(any));
        if (!any) break;
        HPCCG_CUDA(launch_cg64_body(B, g, s));
      }
      HPCCG_CUDA(phase<PhResidual64>(B, g, s));
    } else {
      HPCCG_CUDA(phase<PhOuter64>(B, g, s));
      for (;;) {
        int any = 0;
        HPCCG_CUDA(any_active(any));
        if (!any) break;
        cudaError_t e = precision == HPCCG_PREC_BF16 ? launch_outer_body<__nv_bfloat16>(B, g, s, nullptr, false)
                                                     : launch_outer_body<float>(B, g, s, nullptr, false);
        HPCCG_CUDA(e);
      }
    }
    return HPCCG_OK;
  }
  if (!B->exec[precision] || B->exec_tile[precision] != B->tile_chunks || B->exec_bps[precision] != B->blocks_per_sm ||
      B->exec_tol[precision] != rel_tol || B->exec_maxit[precision] != max_iter ||
      B->exec_kind[precision] != B->spmv_kind) {
    if (B->exec[precision]) cudaGraphExecDestroy(B->exec[precision]);
    B->exec[precision] = nullptr;
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle ho = 0, hi = 0;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&ho, cg, 0, cudaGraphCondAssignDefault);
    g.c_outer = ho;
    g.use_cond = 1;
    if (e == cudaSuccess) e = phase<PhBnorm>(B, g, s);
    if (e == cudaSuccess) e = precision == HPCCG_PREC_FP64 ? phase<PhInit64>(B, g, s) : phase<PhOuter64>(B, g, s);
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams cp = {};
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = ho;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&node, cg, deps, nd, &cp);
    }
    cudaStream_t bs = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      if (precision != HPCCG_PREC_FP64) e = cudaGraphConditionalHandleCreate(&hi, body, 0, 0);
      g.c_inner = hi;
      if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t e1;
        if (precision == HPCCG_PREC_FP64) e1 = launch_cg64_body(B, g, bs);
        else if (precision == HPCCG_PREC_BF16) e1 = launch_outer_body<__nv_bfloat16>(B, g, bs, body, true);
        else e1 = launch_outer_body<float>(B, g, bs, body, true);
        const cudaError_t e2 = cudaStreamEndCapture(bs, &body);
        e = e1 != cudaSuccess ? e1 : e2;
      }
      cudaStreamDestroy(bs);
    }
    if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess && precision == HPCCG_PREC_FP64) e = phase<PhResidual64>(B, g, s);
    cudaGraph_t outg = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &outg);
    if (e == cudaSuccess) e = ee;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&B->exec[precision], outg, 0);
    if (outg) cudaGraphDestroy(outg);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_cuda_error(e, "build batch graph", __FILE__, __LINE__);
    }
    B->exec_tile[precision] = B->tile_chunks;
    B->exec_kind[precision] = B->spmv_kind;
    B->exec_bps[precision] = B->blocks_per_sm;
    B->exec_tol[precision] = rel_tol;
    B->exec_maxit[precision] = max_iter;
  }
  HPCCG_CUDA(cudaGraphLaunch(B->exec[precision], s));
  return HPCCG_OK;
}

__global__ void k_batch_to_lp(const double *src, float *f32, __nv_bfloat16 *b16, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    if (f32) f32[i] = (float)src[i];
    if (b16) b16[i] = __double2bfloat16(src[i]);
  }
}

static int ensure_lp(hpccg_batch *B, int precision) {
  const size_t slots = (size_t)27 * B->npad;
  if (precision == HPCCG_PREC_FP32 && !B->val32) {
    HPCCG_CUDA(cudaMalloc(&B->val32, sizeof(float) * slots));
    k_batch_to_lp<<<B->num_sms * 8, 256, 0, B->stream>>>(B->val, B->val32, nullptr, slots);
  }
  if (precision == HPCCG_PREC_BF16 && !B->val16) {
    HPCCG_CUDA(cudaMalloc(&B->val16, sizeof(__nv_bfloat16) * slots));
    k_batch_to_lp<<<B->num_sms * 8, 256, 0, B->stream>>>(B->val, nullptr, B->val16, slots);
  }
  HPCCG_CUDA(cudaStreamSynchronize(B->stream));
  return HPCCG_OK;
}

// Times one FP64 CG iteration (p update, SpMV + dot, r update) per candidate
// schedule and keeps the fastest.  It runs before a solve copies b and x in,
// on the solver's scratch vectors, with every system's scalars reset before
// each phase so that all systems stay active whatever the data.  Candidates
// differ only in tile size and grid, so the solves they produce are
// bit-identical.
static int autotune(hpccg_batch *B) {
  if (B->tuned) return HPCCG_OK;
  B->tuned = true;
  const int tiles[] = {1, 2, 4, 8};
  const int bps[] = {2, 4, 8};
  float best = 1e30f;
  int bt = 4, bb = 4;
  std::vector<BatchSys> hs(B->nsys);
  for (auto &y : hs) {
    y = BatchSys{};
    y.active = 1;
    y.k = 1;
    y.rtrans = 1.0;
    y.alpha = 0.5;
    y.beta = 0.5;
    y.tol2 = -1.0;  // never converged
  }
  const size_t sys_bytes = sizeof(BatchSys) * B->nsys;
  for (int t : tiles)
    for (int b : bps) {
      int rc = build_tiles(B, t);
      if (rc) return rc;
      B->blocks_per_sm = b;
      BatchArgs g = batch_args(B, HPCCG_PREC_FP64);
      g.max_iter = 1 << 30;
      float ms = 0.f;
      for (int rep = 0; rep < 4; ++rep) {
        if (rep == 1) HPCCG_CUDA(cudaEventRecord(B->ev0, B->stream));
        HPCCG_CUDA(cudaMemcpyAsync(B->sys, hs.data(), sys_bytes, cudaMemcpyHostToDevice, B->stream));
        k_batch_p64<<<grid_of(B), 256, 0, B->stream>>>(g);
        HPCCG_CUDA(cudaGetLastError());
        HPCCG_CUDA(cudaMemcpyAsync(B->sys, hs.data(), sys_bytes, cudaMemcpyHostToDevice, B->stream));
        HPCCG_CUDA(launch_spmv_dot64(B, g, B->stream));
        HPCCG_CUDA(cudaMemcpyAsync(B->sys, hs.data(), sys_bytes, cudaMemcpyHostToDevice, B->stream));
        HPCCG_CUDA(phase<PhUpdate64>(B, g, B->stream));
      }
      HPCCG_CUDA(cudaEventRecord(B->ev1, B->stream));
      HPCCG_CUDA(cudaEventSynchronize(B->ev1));
      HPCCG_CUDA(cudaEventElapsedTime(&ms, B->ev0, B->ev1));
      if (ms < best) {
        best = ms;
        bt = t;
        bb = b;
      }
    }
  B->blocks_per_sm = bb;
  return build_tiles(B, bt);
}

extern "C" int hpccg_batch_set_schedule(hpccg_batch *B, int32_t tile_chunks, int32_t blocks_per_sm) {
  if (!B || tile_chunks < 0 || blocks_per_sm < 0 || tile_chunks > 64 || blocks_per_sm > 16) return HPCCG_ERR_INVALID_ARG;
  if (tile_chunks == 0 || blocks_per_sm == 0) {
    B->tuned = false;
    return HPCCG_OK;
  }
  B->tuned = true;
  B->blocks_per_sm = blocks_per_sm;
  return build_tiles(B, tile_chunks);
}

extern "C" int hpccg_batch_set_spmv(hpccg_batch *B, int32_t kind) {
  if (!B) return HPCCG_ERR_INVALID_ARG;
  if (kind == HPCCG_SPMV_AUTO) kind = HPCCG_SPMV_ELL;
  if (kind != HPCCG_SPMV_ELL && kind != HPCCG_SPMV_STENCIL) return HPCCG_ERR_INVALID_ARG;
  if (kind == HPCCG_SPMV_STENCIL && !B->d_dims) return HPCCG_ERR_UNSUPPORTED;
  if (kind != B->spmv_kind) {
    B->spmv_kind = kind;
    B->tuned = false;  // the schedule is re-timed with the new rows
  }
  return HPCCG_OK;
}

extern "C" int hpccg_batch_get_schedule(const hpccg_batch *B, int32_t *tile_chunks, int32_t *blocks_per_sm) {
  if (!B) return HPCCG_ERR_INVALID_ARG;
  if (tile_chunks) *tile_chunks = B->tile_chunks;
  if (blocks_per_sm) *blocks_per_sm = B->blocks_per_sm;
  return HPCCG_OK;
}

extern "C" int hpccg_batch_spmv(hpccg_batch *B, const double *d_x, double *d_y) {
  if (!B || !d_x || !d_y || d_x == d_y) return HPCCG_ERR_INVALID_ARG;
  BatchArgs g = batch_args(B, HPCCG_PREC_FP64);
  k_batch_spmv<<<grid_of(B), 256, 0, B->stream>>>(g, d_x, d_y);
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaStreamSynchronize(B->stream));
  return HPCCG_OK;
}

// The solve of hpccg_batch_solve; b and x are copied in with `in` and the
// solution out with `out` (device-to-device for device vectors, host-to-device
// and device-to-host for host arrays).
static int batch_solve(hpccg_batch *B, const double *d_b, double *d_x, cudaMemcpyKind in, cudaMemcpyKind out,
                       int32_t precision, double rel_tol, int32_t max_iter, int32_t *iters, double *relres,
                       int32_t *outer) {
  if (!B || !d_b || !d_x || !(rel_tol >= 0.0) || max_iter < 0) return HPCCG_ERR_INVALID_ARG;
  if (precision != HPCCG_PREC_FP64 && precision != HPCCG_PREC_FP32 && precision != HPCCG_PREC_BF16)
    return HPCCG_ERR_INVALID_ARG;
  int rc = autotune(B);
  if (rc) return rc;
  if (precision != HPCCG_PREC_FP64 && B->spmv_kind != HPCCG_SPMV_STENCIL && (rc = ensure_lp(B, precision)))
    return rc;
  const size_t bytes = sizeof(double) * B->npad;
  HPCCG_CUDA(cudaMemcpyAsync(B->b, d_b, bytes, in, B->stream));
  HPCCG_CUDA(cudaMemcpyAsync(B->x, d_x, bytes, in, B->stream));
  HPCCG_CUDA(cudaEventRecord(B->ev0, B->stream));
  const bool eager = getenv("HPCCG_EAGER") && atoi(getenv("HPCCG_EAGER")) != 0;
  rc = run_batch(B, precision, eager, rel_tol, max_iter);
  if (rc) return rc;
  HPCCG_CUDA(cudaEventRecord(B->ev1, B->stream));
  HPCCG_CUDA(cudaMemcpyAsync(d_x, B->x, bytes, out, B->stream));
  std::vector<BatchSys> hs(B->nsys);
  HPCCG_CUDA(cudaMemcpyAsync(hs.data(), B->sys, sizeof(BatchSys) * B->nsys, cudaMemcpyDeviceToHost, B->stream));
  HPCCG_CUDA(cudaStreamSynchronize(B->stream));
  HPCCG_CUDA(cudaEventElapsedTime(&B->last_ms, B->ev0, B->ev1));
  int status = HPCCG_OK;
  for (int s = 0; s < B->nsys; ++s) {
    if (iters) iters[s] = hs[s].iters;
    if (relres) relres[s] = hs[s].relres;
    if (outer) outer[s] = hs[s].outer;
    if (hs[s].status) status = hs[s].status;
    else if (!hs[s].converged && status == HPCCG_OK) status = HPCCG_ERR_NOT_CONVERGED;
  }
  return status;
}

extern "C" int hpccg_batch_solve(hpccg_batch *B, const double *d_b, double *d_x, int32_t precision,
                                 double rel_tol, int32_t max_iter, int32_t *iters, double *relres,
                                 int32_t *outer) {
  return batch_solve(B, d_b, d_x, cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice, precision, rel_tol, max_iter,
                     iters, relres, outer);
}

extern "C" int hpccg_batch_solve_host(hpccg_batch *B, const double *b, double *x, int32_t precision,
                                      double rel_tol, int32_t max_iter, int32_t *iters, double *relres,
                                      int32_t *outer) {
  return batch_solve(B, b, x, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, precision, rel_tol, max_iter, iters,
                     relres, outer);
}

extern "C" int hpccg_batch_last_solve_ms(const hpccg_batch *B, float *ms) {
  if (!B || !ms) return HPCCG_ERR_INVALID_ARG;
  *ms = B->last_ms;
  return HPCCG_OK;
}
