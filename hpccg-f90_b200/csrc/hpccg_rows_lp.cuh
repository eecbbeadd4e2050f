// hpccg_rows_lp.cuh -- low-precision ELL row strategies for the inner solves of
// FP64 iterative refinement.  Values are FP32 or BF16 (a copy of the FP64 ELL
// values), vectors are FP32, each row sum accumulates in FP32 with FMA.
// RPT consecutive rows per thread: slot k of a warp is one contiguous
// 32*RPT*sizeof(value) load plus a 32*RPT*4-byte column-index load.
#pragma once
#include "hpccg_internal.cuh"
#include "hpccg_stencil.cuh"

namespace hpccg {

template <typename VT, int RPT>
struct LpLoad;

template <>
struct LpLoad<float, 1> {
  static __device__ __forceinline__ void vals(const float *p, size_t i, float *v) { v[0] = __ldcs(p + i); }
};
template <>
struct LpLoad<float, 2> {
  static __device__ __forceinline__ void vals(const float *p, size_t i, float *v) {
    const float2 t = __ldcs(reinterpret_cast<const float2 *>(p) + i);
    v[0] = t.x;
    v[1] = t.y;
  }
};
template <>
struct LpLoad<float, 4> {
  static __device__ __forceinline__ void vals(const float *p, size_t i, float *v) {
    const float4 t = __ldcs(reinterpret_cast<const float4 *>(p) + i);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
};
template <>
struct LpLoad<__nv_bfloat16, 1> {
  static __device__ __forceinline__ void vals(const __nv_bfloat16 *p, size_t i, float *v) {
    const unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p) + i);
    v[0] = __uint_as_float((unsigned)u << 16);
  }
};
template <>
struct LpLoad<__nv_bfloat16, 2> {
  static __device__ __forceinline__ void vals(const __nv_bfloat16 *p, size_t i, float *v) {
    const unsigned u = __ldcs(reinterpret_cast<const unsigned *>(p) + i);
    v[0] = __uint_as_float(u << 16);
    v[1] = __uint_as_float(u & 0xffff0000u);
  }
};
template <>
struct LpLoad<__nv_bfloat16, 4> {
  static __device__ __forceinline__ void vals(const __nv_bfloat16 *p, size_t i, float *v) {
    const uint2 u = __ldcs(reinterpret_cast<const uint2 *>(p) + i);
    v[0] = __uint_as_float(u.x << 16);
    v[1] = __uint_as_float(u.x & 0xffff0000u);
    v[2] = __uint_as_float(u.y << 16);
    v[3] = __uint_as_float(u.y & 0xffff0000u);
  }
};

template <int RPT>
__device__ __forceinline__ void lp_cols(const int32_t *p, size_t i, int *c) {
  if constexpr (RPT == 1) {
    c[0] = __ldcs(p + i);
  } else if constexpr (RPT == 2) {
    const int2 t = __ldcs(reinterpret_cast<const int2 *>(p) + i);
    c[0] = t.x;
    c[1] = t.y;
  } else {
    const int4 t = __ldcs(reinterpret_cast<const int4 *>(p) + i);
    c[0] = t.x;
    c[1] = t.y;
    c[2] = t.z;
    c[3] = t.w;
  }
}

// Walks rows in groups of RPT; epi(i, rowsum) stores and returns a dot term.
template <typename VT, int RPT, int W, class Epi>
__device__ __forceinline__ double ell_rows_lp(int n, int npad, const int32_t *__restrict__ col,
                                              const VT *__restrict__ val,
                                              const float *__restrict__ x, Epi &epi) {
  double part = 0.0;
  const int stride = gridDim.x * blockDim.x;
  const int ngroups = (n + RPT - 1) / RPT;
  const size_t slot = (size_t)(npad / RPT);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ngroups; t += stride) {
    float s[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) s[r] = 0.f;
#pragma unroll
    for (int k = 0; k < W; ++k) {
      int c[RPT];
      float v[RPT];
      lp_cols<RPT>(col, (size_t)k * slot + t, c);
      LpLoad<VT, RPT>::vals(val, (size_t)k * slot + t, v);
#pragma unroll
      for (int r = 0; r < RPT; ++r) s[r] = fmaf(v[r], __ldg(x + c[r]), s[r]);
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int i = t * RPT + r;
      if (i < n) part += epi(i, s[r]);
    }
  }
  return part;
}

template <typename VT, int RPT, int MINB>
struct StratLp {
  static constexpr int kMinBlocks = MINB;
  static int grid(const PlaneMap &, const StencilGeom &, int dflt) { return dflt; }
  template <class Epi>
  static __device__ __forceinline__ double rows(int n, int npad, const int32_t *col, const VT *val,
                                                const float *x, Epi &e, const StencilGeom &, const PlaneMap &) {
    return ell_rows_lp<VT, RPT, 27>(n, npad, col, val, x, e);
  }
};

// Matrix-free FP32 rows of the generate_matrix operator (its values 27 and -1
// are exact in FP32 and BF16 alike, so one kernel serves both precisions);
// 3x3 box sums along the plane map, or along the four-column map of
// stencil_rows_boxw<4> (nx a multiple of 4; eight columns measured slower).
// The map comes with the arguments (lp_map on the host).
struct StratLpStencil {
  static constexpr int kMinBlocks = 4;
  static int grid(const PlaneMap &m, const StencilGeom &, int dflt) { return m.plane > 0 ? plane_grid(m) : dflt; }
  template <class Epi>
  static __device__ __forceinline__ double rows(int n, int, const int32_t *, const float *, const float *x,
                                                Epi &e, const StencilGeom &g, const PlaneMap &m) {
    if (m.cols == 4) return stencil_rows_boxw<4>(g, m, x, e);
    return m.plane > 0 ? stencil_rows_box(g, m, x, e) : stencil_rows<float>(n, g, m, x, e);
  }
};

}  // namespace hpccg
