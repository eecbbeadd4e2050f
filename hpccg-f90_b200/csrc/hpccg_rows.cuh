// hpccg_rows.cuh -- row strategies of the FP64 SpMV (MPI/src/SparseMatrix.F90:213-232).
//
// Every strategy walks the rows of A, forms rowsum_i = sum_k val_k * x[col_k],
// and hands (i, rowsum_i) to an epilogue functor that stores the result and
// returns this row's contribution to a fused dot product.
//
//  * ell_rows<W,RPT>: one thread per row (RPT = 1) or per row pair (RPT = 2)
//    over the column-major ELL copy.  Slot k of 32 consecutive rows is one
//    256-byte (RPT=1) or 512-byte (RPT=2) coalesced load; the x gather for a
//    stencil slot hits 32 consecutive x entries.  The sum runs k = 0..W-1 in
//    order with separately rounded multiply and add, exactly the reference's
//    `rowsum = rowsum + values(k)*x(colindex(k))`, so y is bit-identical to
//    the reference's spmv.  Matrix streams use evict-first loads so that L2
//    keeps x.
//  * csr_vector_rows<LPR>: LPR lanes per CSR row (LPR = 32 is warp-per-row),
//    lane-strided loads, butterfly shuffle reduction.  Reassociates the sum.
//  * stencil_rows (hpccg_stencil.cuh): matrix-free, for a context whose CSR
//    was checked equal to generate_matrix(nx,ny,nz); bit-identical to ELL
//    (both follow the same plane map of rows to threads).
#pragma once
#include "hpccg_internal.cuh"
#include "hpccg_stencil.cuh"
#include "hpccg_stencil_tma64.cuh"

// z planes per block of the FP64 tile map: at most this many while the grid
// gives every SM four blocks or more, down to 8 on small grids; more when the
// blocks would exceed the reduction scratch.
#ifndef HPCCG_TILE_ZC
#define HPCCG_TILE_ZC 16
#endif

namespace hpccg {

__device__ __forceinline__ double mul_add(double s, double v, double x) {
  return __dadd_rn(s, __dmul_rn(v, x));  // no contraction: reference rounding
}

// Calls body(i) for the calling thread's rows, in order: the plane map when
// it is in use (hpccg_stencil.cuh), else grid-stride rows.
template <class Body>
__device__ __forceinline__ void thread_rows(int n, const PlaneMap &m, Body &&body) {
  if (m.tiles_x > 0) {  // the column pair of a tile, the order of stencil_rows_tma64ref
    const TileSpan sp = tile_span(m, n / m.plane);
    if (!sp.rows) return;
    for (int z = sp.z0; z < sp.z1; ++z) {
      body(sp.c + z * m.plane);
      body(sp.c + m.nx + z * m.plane);
    }
    return;
  }
  if (m.plane > 0) {
    const PlaneSpan sp = plane_span(m, n / m.plane);
    if (m.ry == 2) {  // the column pair (x, y), (x, y+1), the order of stencil_column2
      for (int z = sp.z0; z < sp.z1; ++z) {
        body(sp.c + z * m.plane);
        body(sp.c + m.nx + z * m.plane);
      }
      return;
    }
    for (int z = sp.z0; z < sp.z1; ++z) body(sp.c + z * m.plane);
    return;
  }
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) body(i);
}

template <int W, int RPT, int U, class Epi>
__device__ __forceinline__ double ell_rows(int n, int npad, const int32_t *__restrict__ col,
                                           const double *__restrict__ val,
                                           const double *__restrict__ x, Epi &epi, const PlaneMap &m) {
  static_assert(W % U == 0, "slot chunk must divide the ELL width");
  double part = 0.0;
  if constexpr (RPT == 1) {
    thread_rows(n, m, [&](int i) {
      double s = 0.0;
#pragma unroll
      for (int k0 = 0; k0 < W; k0 += U) {
        int32_t c[U];
        double v[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
          c[k] = __ldcs(col + (size_t)(k0 + k) * npad + i);
          v[k] = __ldcs(val + (size_t)(k0 + k) * npad + i);
        }
#pragma unroll
        for (int k = 0; k < U; ++k) s = mul_add(s, v[k], __ldg(x + c[k]));
      }
      part = __dadd_rn(part, epi(i, s));
    });
  } else {
    const int stride = gridDim.x * blockDim.x;
    const int half = npad >> 1;
    const int npairs = (n + 1) >> 1;
    const int2 *col2 = reinterpret_cast<const int2 *>(col);
    const double2 *val2 = reinterpret_cast<const double2 *>(val);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += stride) {
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int k0 = 0; k0 < W; k0 += U) {
        int2 c[U];
        double2 v[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
          c[k] = __ldcs(col2 + (size_t)(k0 + k) * half + t);
          v[k] = __ldcs(val2 + (size_t)(k0 + k) * half + t);
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
          s0 = mul_add(s0, v[k].x, __ldg(x + c[k].x));
          s1 = mul_add(s1, v[k].y, __ldg(x + c[k].y));
        }
      }
      const int i0 = 2 * t;
      part = __dadd_rn(part, epi(i0, s0));
      if (i0 + 1 < n) part = __dadd_rn(part, epi(i0 + 1, s1));
    }
  }
  return part;
}

// Runtime-width variant for ELL widths other than the compiled ones.
template <class Epi>
__device__ __forceinline__ double ell_rows_dyn(int n, int npad, int W,
                                               const int32_t *__restrict__ col,
                                               const double *__restrict__ val,
                                               const double *__restrict__ x, Epi &epi, const PlaneMap &m) {
  double part = 0.0;
  thread_rows(n, m, [&](int i) {
    double s = 0.0;
#pragma unroll 4
    for (int k = 0; k < W; ++k)
      s = mul_add(s, __ldcs(val + (size_t)k * npad + i), __ldg(x + __ldcs(col + (size_t)k * npad + i)));
    part = __dadd_rn(part, epi(i, s));
  });
  return part;
}

template <int LPR, class Epi>
__device__ __forceinline__ double csr_vector_rows(int n, const int32_t *__restrict__ rowptr,
                                                  const int32_t *__restrict__ col,
                                                  const double *__restrict__ val,
                                                  const double *__restrict__ x, Epi &epi) {
  constexpr int RPW = 32 / LPR;  // rows per warp
  double part = 0.0;
  const int lane = threadIdx.x & 31;
  const int sub = lane / LPR, sl = lane % LPR;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = warp * RPW; base < n; base += nwarps * RPW) {  // warp-uniform trip count
    const int row = base + sub;
    double s = 0.0;
    if (row < n) {
      const int a = __ldg(rowptr + row), e = __ldg(rowptr + row + 1);
      for (int j = a + sl; j < e; j += LPR) s = mul_add(s, __ldcs(val + j), __ldg(x + __ldcs(col + j)));
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
    if (sl == 0 && row < n) part = __dadd_rn(part, epi(row, s));
  }
  return part;
}

// ---- epilogues --------------------------------------------------------------
// The three-argument forms receive x_i (the matrix-free walk has it at hand).
struct EpiStore {  // y = A x
  double *y;
  __device__ __forceinline__ double operator()(int i, double s) const {
    y[i] = s;
    return 0.0;
  }
  __device__ __forceinline__ double operator()(int i, double s, double) const { return (*this)(i, s); }
};
struct EpiDot {  // Ap = A p, contribution p_i * Ap_i
  const double *p;
  double *y;
  __device__ __forceinline__ double operator()(int i, double s) const {
    y[i] = s;
    return __dmul_rn(__ldg(p + i), s);
  }
  __device__ __forceinline__ double operator()(int i, double s, double pi) const {
    y[i] = s;
    return __dmul_rn(pi, s);
  }
};
struct EpiResidual {  // r = 1*b + (-1)*(A x), contribution r_i^2
  const double *b;
  double *r;
  __device__ __forceinline__ double operator()(int i, double s) const {
    const double ri = __dsub_rn(__ldg(b + i), s);
    r[i] = ri;
    return __dmul_rn(ri, ri);
  }
  __device__ __forceinline__ double operator()(int i, double s, double) const { return (*this)(i, s); }
};

// Arguments every row strategy may need.
struct SpmvArgs {
  int kind;   // HPCCG_SPMV_ELL / ELL2 / CSR_VECTOR / STENCIL
  int param;  // lanes per row for CSR_VECTOR
  int n, npad, W;
  const int32_t *rowptr, *col, *ell_col;
  const double *val, *ell_val;
  StencilGeom geom;  // grid of generate_matrix (STENCIL only)
  PlaneMap pm;       // row map of ELL (one row per thread) and STENCIL when the grid is known
  // STENCIL under the tile map: tensor maps of the two vectors tma_vec[0..1],
  // whose SpMVs read x by TMA (tma_ok); other vectors use plain loads.  The
  // kernels take SpmvArgs as a __grid_constant__ parameter, so the TMA reads
  // the maps from parameter space.
  CUtensorMap tmap[2];
  const double *tma_vec[2];
  int tma_ok;
  int *status;  // where a TMA walk records HPCCG_ERR_TIMEOUT
};

// Launch grid of a strategy that follows the plane map when it is in use.
inline int plane_or(const PlaneMap &m, int dflt) { return m.plane > 0 ? plane_grid(m) : dflt; }

// Strategy tags: each kernel is compiled once per strategy and the host picks
// the instantiation.  kMinBlocks feeds __launch_bounds__: with 2 resident
// blocks per SM ptxas keeps all 27 slot loads of a row in flight (~120
// registers); with 8 it interleaves loads and gathers at 32 registers and
// relies on occupancy instead.  Strategies with the same RPT map rows to
// threads identically, so they give bit-identical results (fused dots too);
// one row per thread (ELL, STENCIL) follows the plane map when the grid of
// the matrix is known.
template <int MINB>
struct StratEll1 {
  static constexpr int kMinBlocks = MINB;
  static int grid(const SpmvArgs &a, int dflt) { return plane_or(a.pm, dflt); }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return ell_rows<27, 1, 27>(a.n, a.npad, a.ell_col, a.ell_val, x, e, a.pm);
  }
};
template <int MINB>
struct StratEll2 {
  static constexpr int kMinBlocks = MINB;
  static int grid(const SpmvArgs &, int dflt) { return dflt; }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return ell_rows<27, 2, 9>(a.n, a.npad, a.ell_col, a.ell_val, x, e, a.pm);
  }
};
struct StratEllDyn {
  static constexpr int kMinBlocks = 4;
  static int grid(const SpmvArgs &a, int dflt) { return plane_or(a.pm, dflt); }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return ell_rows_dyn(a.n, a.npad, a.W, a.ell_col, a.ell_val, x, e, a.pm);
  }
};
template <int LPR>
struct StratCsr {
  static constexpr int kMinBlocks = 4;
  static int grid(const SpmvArgs &, int dflt) { return dflt; }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return csr_vector_rows<LPR>(a.n, a.rowptr, a.col, a.val, x, e);
  }
};

struct StratStencil {
  static constexpr int kMinBlocks = 4;
  static int grid(const SpmvArgs &a, int dflt) { return plane_or(a.pm, dflt); }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return stencil_rows<double>(a.n, a.geom, a.pm, x, e);
  }
};
// The same rows and sums with x streamed by TMA (tile map; the host selects it
// only for x = tma_vec[0] or tma_vec[1], whose tensor maps a.tmap holds).
struct StratStencilTma {
  static constexpr int kMinBlocks = 4;
  static int grid(const SpmvArgs &a, int dflt) { return plane_or(a.pm, dflt); }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return stencil_rows_tma64ref(a.geom, a.pm, &a.tmap[x == a.tma_vec[0] ? 0 : 1], e, a.status);
  }
};

// FP64 box walk with four columns per thread (the outer residual of the
// refinement; a.pm must be a boxw_map(4, ...) map).
struct StratStencilBox64 {
  static constexpr int kMinBlocks = 2;
  static int grid(const SpmvArgs &a, int dflt) { return plane_or(a.pm, dflt); }
  template <class Epi>
  static __device__ __forceinline__ double rows(const SpmvArgs &a, const double *x, Epi &e) {
    return stencil_rows_box64x4(a.geom, a.pm, x, e);
  }
};

// Resident-block hints offered for the ELL strategies (the `param` of
// hpccg_gpu_set_spmv for HPCCG_SPMV_ELL / HPCCG_SPMV_ELL2).
constexpr int kEllMinBlocks[4] = {2, 3, 4, 8};

// Calls f(Strat{}) with the strategy the arguments select (host side); x, the
// vector the SpMV reads, selects the TMA walk when its tensor map exists.
template <class F>
inline int dispatch_strategy(const SpmvArgs &a, F &&f, const double *x = nullptr) {
  if (a.kind == HPCCG_SPMV_STENCIL) {
    if (x && a.tma_ok && a.pm.tiles_x > 0 && (x == a.tma_vec[0] || x == a.tma_vec[1])) return f(StratStencilTma{});
    return f(StratStencil{});
  }
  if (a.kind == HPCCG_SPMV_CSR_VECTOR) {
    switch (a.param) {
      case 4: return f(StratCsr<4>{});
      case 8: return f(StratCsr<8>{});
      case 16: return f(StratCsr<16>{});
      default: return f(StratCsr<32>{});
    }
  }
  if (a.W != 27) return f(StratEllDyn{});
  if (a.kind == HPCCG_SPMV_ELL2) {
    switch (a.param) {
      case 2: return f(StratEll2<2>{});
      case 3: return f(StratEll2<3>{});
      case 8: return f(StratEll2<8>{});
      default: return f(StratEll2<4>{});
    }
  }
  switch (a.param) {
    case 2: return f(StratEll1<2>{});
    case 3: return f(StratEll1<3>{});
    case 8: return f(StratEll1<8>{});
    default: return f(StratEll1<4>{});
  }
}

// Row map of the FP64 kernels of a context whose grid is known: the tile map
// when nx and ny are even (nx even: the TMA walk's tensor map), else the
// two-line plane map.
inline PlaneMap fp64_map(int nx, int ny, int nz, int num_sms) {
  if (nx % 2 == 0) {
    int zc = HPCCG_TILE_ZC;
    const int64_t per_plane = (int64_t)((nx + kTileX - 1) / kTileX) * ((ny + kTileY - 1) / kTileY);
    while (zc > 8 && per_plane * ((nz + zc - 1) / zc) < 4 * (int64_t)num_sms) zc /= 2;
    const PlaneMap t = tile_map(nx, ny, nz, kMaxPartials, zc);
    if (t.plane > 0) return t;
  }
  return plane_map(nx, ny, nz, kMaxPartials, 2);
}

inline SpmvArgs spmv_args(const hpccg_ctx *c) {
  SpmvArgs a;
  a.kind = c->spmv_kind == HPCCG_SPMV_AUTO ? HPCCG_SPMV_ELL : c->spmv_kind;
  a.param = c->spmv_kind == HPCCG_SPMV_AUTO ? 4 : c->spmv_param;
  if (a.kind == HPCCG_SPMV_STENCIL && !c->gx) a.kind = HPCCG_SPMV_ELL;
  if (!c->d_ell_col && a.kind != HPCCG_SPMV_CSR_VECTOR && a.kind != HPCCG_SPMV_STENCIL) {
    a.kind = HPCCG_SPMV_CSR_VECTOR;
    a.param = 32;
  }
  a.n = c->nrow;
  a.npad = c->npad;
  a.W = c->ell_width;
  a.rowptr = c->d_rowptr;
  a.col = c->d_col;
  a.val = c->d_val;
  a.ell_col = c->d_ell_col;
  a.ell_val = c->d_ell_val;
  a.geom = StencilGeom{c->gx, c->gy, c->gz};
  a.pm = c->gx ? fp64_map(c->gx, c->gy, c->gz, c->num_sms) : PlaneMap{0, 0, 0, 1, 1, 0};
  a.tma_ok = a.pm.tiles_x > 0 && c->tmaps_ok;
  if (a.tma_ok) {
    a.tmap[0] = c->tmaps[0];
    a.tmap[1] = c->tmaps[1];
  }
  a.tma_vec[0] = c->d_p;
  a.tma_vec[1] = c->d_x;
  a.status = &c->d_state->status;
  return a;
}

}  // namespace hpccg
