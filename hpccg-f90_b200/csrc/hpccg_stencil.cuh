// hpccg_stencil.cuh -- matrix-free SpMV with the operator of generate_matrix
// (MPI/src/SparseMatrix.F90:138-159): 27.0 on the diagonal, -1.0 for every
// in-grid neighbour of the 3x3x3 stencil, nothing for neighbours outside the
// grid.  Only x and y cross HBM; the matrix is never read.
//
// Row i's terms are added in the reference's k order (sz, then sy, then sx,
// each -1..1, which is ascending column order): rowsum = rowsum + v*x(col)
// with v*x exact for v = -1 (so the add equals rowsum - x(col)) and
// __dmul_rn(27, x(i)) for the diagonal.  A neighbour outside the grid
// subtracts +0.0, which leaves the sum unchanged: the sum starts at +0.0 and
// round-to-nearest never produces -0.0 from it.  So the FP64 row sums are
// bit-identical to the CSR/ELL kernels'.
//
// Row-to-thread map ("plane map", used when the grid is known): thread t
// owns the grid column c = t mod nx*ny and walks z through one chunk of zc
// planes, rows c + z*nx*ny for z in [q*zc, min(nz, (q+1)*zc)), q = t div
// nx*ny.  Consecutive threads own consecutive rows (coalesced), and a thread
// keeps what it needs of planes z-1, z, z+1 in registers, so each row takes
// 9 new values instead of 27.  The FP64 kernels of a context with an even ny
// use the two-line form (ry = 2): thread t owns the columns (x, y) and
// (x, y+1) of an even line y, so twelve loads a plane serve two rows (6 a
// row); at 256^3 the matrix-free FP64 SpMV went 0.109 -> 0.095 ms with it.
// With nx and ny even the FP64 kernels use the tile map below instead (32 x
// 16 columns a block, the same column pairs), whose rectangles a TMA box can
// feed (hpccg_stencil_tma64.cuh).  The ELL kernel uses the same map for the
// same context, so fused dot products -- and whole CG runs -- are
// bit-identical between the two.
#pragma once
#include <algorithm>

#include "hpccg_internal.cuh"

namespace hpccg {

struct StencilGeom {
  int nx, ny, nz;
};

struct PlaneMap {
  int plane;  // nx*ny rows per z plane (divided by cols); 0 = map not in use (grid-stride rows)
  int zc;     // planes per thread
  int nzc;    // z chunks
  int cols;   // consecutive grid columns per thread (0 or 1: one; 4: the FP32 box walk)
  int ry;     // plane map: grid lines per thread (0 or 1: one; 2: lines y and y+1, y even)
  int nx;     // plane map with ry = 2: the grid's nx
  int tiles_x, tiles_y;  // > 0: tile map (below), tiles per plane
};

// Tile map of the FP64 walks (ry = 2): block b owns the kTileX x kTileY
// columns of tile b mod (tiles_x*tiles_y) and planes [q*zc, (q+1)*zc) of
// chunk q = b div (tiles_x*tiles_y); thread t owns column x = x0 + t mod
// kTileX of the even line y = y0 + 2 (t div kTileX) and of line y+1.  A warp
// is one 32-column line pair, so loads stay coalesced, and a block's columns
// form the rectangle that one TMA box (plus halo) covers.
constexpr int kTileX = 32, kTileY = 2 * (kBlock / kTileX);

// Host: the plane map for a grid, with at most `max_blocks` blocks of kBlock
// threads (the reduction scratch holds one partial per block).  Chunks of at
// least 16 planes keep the per-thread start-up (two extra planes) small.
inline PlaneMap plane_map(int nx, int ny, int nz, int max_blocks, int ry_max = 1) {
  PlaneMap m{0, 0, 0, 1, 1, nx};
  if (nx < 1 || ny < 1 || nz < 1) return m;
  const int64_t plane = (int64_t)nx * ny;
  const int ry = (ry_max >= 2 && ny % 2 == 0) ? 2 : 1;
  for (int zc = 16;; zc *= 2) {
    const int64_t nzc = (nz + zc - 1) / zc;
    const int64_t blocks = (plane / ry * nzc + kBlock - 1) / kBlock;
    if (blocks <= max_blocks / 2 || (zc >= nz && blocks <= max_blocks)) {
      m.plane = (int)plane;
      m.zc = zc;
      m.nzc = (int)nzc;
      m.ry = ry;
      return m;
    }
    if (zc >= nz) return m;  // one plane alone needs too many threads
  }
}
// Host: the tile map for a grid with an even ny, z chunks of zc planes (more
// when the blocks would outnumber max_blocks); plane = 0 when no tile map fits.
inline PlaneMap tile_map(int nx, int ny, int nz, int max_blocks, int zc) {
  PlaneMap m{0, 0, 0, 1, 1, nx, 0, 0};
  if (nx < 1 || ny < 2 || ny % 2 || nz < 1 || zc < 1) return m;
  const int64_t tx = (nx + kTileX - 1) / kTileX, ty = (ny + kTileY - 1) / kTileY;
  for (zc = std::min(zc, nz);; zc = std::min(2 * zc, nz)) {
    const int64_t nzc = (nz + zc - 1) / zc;
    if (tx * ty * nzc <= max_blocks) {
      m.plane = nx * ny;
      m.zc = zc;
      m.nzc = (int)nzc;
      m.ry = 2;
      m.tiles_x = (int)tx;
      m.tiles_y = (int)ty;
      return m;
    }
    if (zc >= nz) return m;
  }
}

// Threads of one z chunk: one per column (or column group), or per column pair in y.
__host__ __device__ __forceinline__ int64_t plane_threads(const PlaneMap &m) {
  return m.ry == 2 ? m.plane / 2 : m.plane;
}
inline int plane_grid(const PlaneMap &m) {
  if (m.tiles_x > 0) return m.tiles_x * m.tiles_y * m.nzc;
  return (int)((plane_threads(m) * m.nzc + kBlock - 1) / kBlock);
}

// The rows of the calling thread under the map: column c, planes [z0, z1).
struct PlaneSpan {
  int c, z0, z1;
};
__device__ __forceinline__ PlaneSpan plane_span(const PlaneMap &m, int nz) {
  PlaneSpan s{0, 0, 0};
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t tpc = plane_threads(m);
  if (t >= tpc * m.nzc) return s;
  const int q = (int)(t / tpc);
  const int u = (int)(t - (int64_t)q * tpc);
  // ry = 2: consecutive threads own consecutive x of one even line y (and line y+1)
  s.c = m.ry == 2 ? (u / m.nx) * 2 * m.nx + u % m.nx : u;
  s.z0 = q * m.zc;
  s.z1 = min(nz, s.z0 + m.zc);
  return s;
}

// The calling thread's rows under a tile map: columns c and c + nx (c at an
// even line y), planes [z0, z1); rows = false for a thread whose column lies
// outside the grid (a partial tile at the x or y face).  x0, y0: the tile.
struct TileSpan {
  int c, z0, z1, x0, y0;
  bool rows;
};
__device__ __forceinline__ TileSpan tile_span(const PlaneMap &m, int nz) {
  TileSpan s;
  const int per = m.tiles_x * m.tiles_y;
  const int q = blockIdx.x / per, tile = blockIdx.x - q * per;
  s.x0 = (tile % m.tiles_x) * kTileX;
  s.y0 = (tile / m.tiles_x) * kTileY;
  const int x = s.x0 + (int)threadIdx.x % kTileX, y = s.y0 + 2 * ((int)threadIdx.x / kTileX);
  s.rows = x < m.nx && y < m.plane / m.nx;  // ny even: line y+1 is inside too
  s.c = y * m.nx + x;
  s.z0 = q * m.zc;
  s.z1 = min(nz, s.z0 + m.zc);
  return s;
}

// One row from 27 loads, row i at grid position (ix, iy, iz).
template <typename Real>
__device__ __forceinline__ Real stencil_row_at(int i, int ix, int iy, int iz, const StencilGeom &g,
                                               const Real *__restrict__ x) {
  const int nxy = g.nx * g.ny;
  const bool has_l = ix > 0, has_r = ix < g.nx - 1;
  Real s = Real(0);
#pragma unroll
  for (int sz = -1; sz <= 1; ++sz) {
#pragma unroll
    for (int sy = -1; sy <= 1; ++sy) {
      const bool line = (unsigned)(iz + sz) < (unsigned)g.nz && (unsigned)(iy + sy) < (unsigned)g.ny;
      const int j = i + sz * nxy + sy * g.nx;
      const Real l = (line && has_l) ? __ldg(x + j - 1) : Real(0);
      const Real c = line ? __ldg(x + j) : Real(0);
      const Real r = (line && has_r) ? __ldg(x + j + 1) : Real(0);
      if constexpr (sizeof(Real) == 8) {
        s = __dsub_rn(s, l);
        s = (sz == 0 && sy == 0) ? __dadd_rn(s, __dmul_rn(27.0, c)) : __dsub_rn(s, c);
        s = __dsub_rn(s, r);
      } else {
        s -= l;
        s = (sz == 0 && sy == 0) ? fmaf(27.f, c, s) : s - c;
        s -= r;
      }
    }
  }
  return s;
}
// FP32 row from 27 loads as 28 x_i - (3-point line sums, 3-line box sums,
// 3-plane sum): the same value as the reference-order sum up to FP32 rounding,
// with a dependency depth of 7 instead of 27 (for rows formed one after
// another by a thread).
__device__ __forceinline__ float stencil_row_box(int i, const StencilGeom &g, const float *__restrict__ x) {
  const int nxy = g.nx * g.ny;
  const int iz = i / nxy, rem = i - iz * nxy;
  const int iy = rem / g.nx, ix = rem - iy * g.nx;
  const bool has_l = ix > 0, has_r = ix < g.nx - 1;
  float pl[3];
#pragma unroll
  for (int sz = -1; sz <= 1; ++sz) {
    float ln[3];
#pragma unroll
    for (int sy = -1; sy <= 1; ++sy) {
      const bool line = (unsigned)(iz + sz) < (unsigned)g.nz && (unsigned)(iy + sy) < (unsigned)g.ny;
      const int j = i + sz * nxy + sy * g.nx;
      const float l = (line && has_l) ? __ldg(x + j - 1) : 0.f;
      const float c = line ? __ldg(x + j) : 0.f;
      const float r = (line && has_r) ? __ldg(x + j + 1) : 0.f;
      ln[sy + 1] = (l + c) + r;
    }
    pl[sz + 1] = (ln[0] + ln[1]) + ln[2];
  }
  return fmaf(28.f, __ldg(x + i), -((pl[0] + pl[1]) + pl[2]));
}

// Grid-stride form (any row order).
template <typename Real>
__device__ __forceinline__ Real stencil_row(int i, const StencilGeom &g, const Real *__restrict__ x) {
  const int nxy = g.nx * g.ny;
  const int iz = i / nxy, rem = i - iz * nxy;
  const int iy = rem / g.nx, ix = rem - iy * g.nx;
  return stencil_row_at<Real>(i, ix, iy, iz, g, x);
}

// Bit j = (sy+1)*3 + (sx+1) set when neighbour (sy, sx) of column (ix, iy)
// lies inside the grid.
__device__ __forceinline__ unsigned stencil_mask(const StencilGeom &g, int ix, int iy) {
  unsigned mask = 0;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    const int yy = iy + j / 3 - 1, xx = ix + j % 3 - 1;
    if ((unsigned)yy < (unsigned)g.ny && (unsigned)xx < (unsigned)g.nx) mask |= 1u << j;
  }
  return mask;
}

// Loads the 3x3 neighbourhood (sy, sx order) of the thread's column in the
// plane that `p` points into (p = &x[column + z*plane]); `mask` bit j clear
// (or zin false) gives 0 for neighbour j, which lies outside the grid.
template <typename Real>
__device__ __forceinline__ void stencil_plane(const Real *__restrict__ p, int nx, unsigned mask, bool zin, Real *v) {
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    const int off = (j / 3 - 1) * nx + (j % 3 - 1);
    v[j] = (zin && ((mask >> j) & 1u)) ? __ldg(p + off) : Real(0);
  }
}

// The row sum split at the plane boundaries, term for term the reference's
// order: lead = the nine terms of plane z-1 from 0, mid = s followed by the
// nine of plane z (27 x_i at the centre), end = s followed by the nine of
// plane z+1; a row is stencil_end(stencil_mid(stencil_lead(a), b), c).
template <typename Real>
__device__ __forceinline__ Real stencil_lead(const Real *a) {
  Real s = Real(0);
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    if constexpr (sizeof(Real) == 8)
      s = __dsub_rn(s, a[j]);
    else
      s -= a[j];
  }
  return s;
}
template <typename Real>
__device__ __forceinline__ Real stencil_mid(Real s, const Real *b) {
  if constexpr (sizeof(Real) == 8) {
#pragma unroll
    for (int j = 0; j < 9; ++j) s = j == 4 ? __dadd_rn(s, __dmul_rn(27.0, b[j])) : __dsub_rn(s, b[j]);
  } else {
#pragma unroll
    for (int j = 0; j < 9; ++j) s = j == 4 ? fmaf(27.f, b[j], s) : s - b[j];
  }
  return s;
}
template <typename Real>
__device__ __forceinline__ Real stencil_end(Real s, const Real *c) {
  if constexpr (sizeof(Real) == 8) {
#pragma unroll
    for (int j = 0; j < 9; ++j) s = __dsub_rn(s, c[j]);
  } else {
#pragma unroll
    for (int j = 0; j < 9; ++j) s -= c[j];
  }
  return s;
}

// FP32 rows of the plane-map walk from 3x3 box sums: y_i = 28 x_i - (sum of
// the 27 values of the 3x3x3 neighbourhood, self included), the box sum of
// each plane formed once and used by the three rows that need it.  This
// reassociates the row sum (for the low-precision inner solves only).  Loads
// are unconditional from clamped addresses and weighted by 0/1 instead of
// predicated (exact: 0*v = 0 for the finite vectors of a solve).
template <class Epi>
__device__ __forceinline__ double stencil_rows_box(const StencilGeom &g, const PlaneMap &m,
                                                   const float *__restrict__ x, Epi &epi) {
  double part = 0.0;
  const PlaneSpan sp = plane_span(m, g.nz);
  if (sp.z0 >= sp.z1) return part;
  const int iy = sp.c / g.nx, ix = sp.c - iy * g.nx;
  const int dl = ix > 0 ? -1 : 0, dr = ix < g.nx - 1 ? 1 : 0;
  const float wl = (float)(-dl), wr = (float)dr;
  const int ylo = iy > 0 ? -g.nx : 0, yhi = iy < g.ny - 1 ? g.nx : 0;
  const float wlo = iy > 0 ? 1.f : 0.f, whi = iy < g.ny - 1 ? 1.f : 0.f;
  const float *pc = x + sp.c;
  // box sum of plane z (zero outside [0, nz)); center = x of the column
  auto box = [&](int z, float &center) {
    const bool zin = (unsigned)z < (unsigned)g.nz;
    const float *p = pc + (int64_t)(zin ? z : 0) * m.plane;
    const float *q0 = p + ylo, *q2 = p + yhi;
    const float c1 = __ldg(p);
    float t1 = fmaf(wl, __ldg(p + dl), c1);
    t1 = fmaf(wr, __ldg(p + dr), t1);
    float t0 = fmaf(wl, __ldg(q0 + dl), __ldg(q0));
    t0 = fmaf(wr, __ldg(q0 + dr), t0);
    float t2 = fmaf(wl, __ldg(q2 + dl), __ldg(q2));
    t2 = fmaf(wr, __ldg(q2 + dr), t2);
    const float s = fmaf(wlo, t0, fmaf(whi, t2, t1));
    center = c1;
    return zin ? s : 0.f;
  };
  float xc, xn, unused;
  float bm = box(sp.z0 - 1, unused), b0 = box(sp.z0, xc);
  for (int z = sp.z0; z < sp.z1; ++z) {
    const float bp = box(z + 1, xn);
    part += epi(sp.c + z * m.plane, fmaf(28.f, xc, -((bm + b0) + bp)), xc);
    bm = b0;
    b0 = bp;
    xc = xn;
  }
  return part;
}

// FP32 box walk with W = 4 or 8 consecutive columns per thread (nx a multiple
// of W): per plane and grid line W/4 aligned 16-byte loads of the columns plus
// the two x neighbours, so a row costs well under 2 loads and ~8 adds.  Its own
// map: thread t owns columns W*(t mod nx*ny/W) .. +W-1 of one z chunk.
// Host: the map of the W-column walk.  The z range of each column is split so
// that all threads are resident at once (one wave): a thread's chunk is then
// as long as possible, which keeps the two extra planes of its start small.
inline PlaneMap boxw_map(int W, int nx, int ny, int nz, int64_t resident_threads) {
  PlaneMap q{0, 0, 0, W};
  if (nx < 1 || ny < 1 || nz < 1 || nx % W) return q;
  const int64_t cols = (int64_t)nx * ny / W;
  const int64_t k = std::max<int64_t>(1, std::min<int64_t>(nz, resident_threads / cols));
  const int zc = (int)((nz + k - 1) / k);
  const int nzc = (nz + zc - 1) / zc;
  if (cols * nzc > (int64_t)kMaxPartials * kBlock) return q;  // keep the reduction scratch
  q.plane = (int)cols;
  q.zc = zc;
  q.nzc = nzc;
  return q;
}

template <int W, class Epi>
__device__ __forceinline__ double stencil_rows_boxw(const StencilGeom &g, const PlaneMap &q,
                                                    const float *__restrict__ x, Epi &epi) {
  static_assert(W % 4 == 0, "whole 16-byte loads");
  double part = 0.0;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)q.plane * q.nzc) return part;
  const int qz = (int)(t / q.plane);
  const int c0 = W * (int)(t - (int64_t)qz * q.plane);  // first of the W columns
  const int z0 = qz * q.zc, z1 = min(g.nz, z0 + q.zc);
  const int iy = c0 / g.nx, ix0 = c0 - iy * g.nx;
  const int plane = W * q.plane;
  const int dl = ix0 > 0 ? -1 : 0, dr = ix0 + W < g.nx ? W : W - 1;
  const float wl = ix0 > 0 ? 1.f : 0.f, wr = ix0 + W < g.nx ? 1.f : 0.f;
  const int ylo = iy > 0 ? -g.nx : 0, yhi = iy < g.ny - 1 ? g.nx : 0;
  const float wlo = iy > 0 ? 1.f : 0.f, whi = iy < g.ny - 1 ? 1.f : 0.f;
  const float *pc = x + c0;
  // 3-point line sums of the W columns of one grid line; v = the line's values
  auto line = [&](const float *p, float *v, float *s) {
#pragma unroll
    for (int k = 0; k < W / 4; ++k) {
      const float4 u = __ldg(reinterpret_cast<const float4 *>(p) + k);
      v[4 * k] = u.x;
      v[4 * k + 1] = u.y;
      v[4 * k + 2] = u.z;
      v[4 * k + 3] = u.w;
    }
    const float l = wl * __ldg(p + dl), r = wr * __ldg(p + dr);
#pragma unroll
    for (int j = 0; j < W; ++j) s[j] = ((j > 0 ? v[j - 1] : l) + v[j]) + (j < W - 1 ? v[j + 1] : r);
  };
  // 3x3 box sums of plane z for the W columns (zero outside [0, nz)); v = the columns' x
  auto box = [&](int z, float *b, float *v) {
    const bool zin = (unsigned)z < (unsigned)g.nz;
    const float *p = pc + (int64_t)(zin ? z : 0) * plane;
    float s0[W], s1[W], s2[W], u[W];
    line(p + ylo, u, s0);
    line(p, v, s1);
    line(p + yhi, u, s2);
    const float wz = zin ? 1.f : 0.f;
#pragma unroll
    for (int j = 0; j < W; ++j) b[j] = wz * fmaf(wlo, s0[j], fmaf(whi, s2[j], s1[j]));
  };
  float bm[W], b0[W], bp[W], vm[W], v0[W], vp[W];
  box(z0 - 1, bm, vm);
  box(z0, b0, v0);
  for (int z = z0; z < z1; ++z) {
    box(z + 1, bp, vp);
#pragma unroll
    for (int k = 0; k < W / 4; ++k) {
      float4 y, xv;
      y.x = fmaf(28.f, v0[4 * k], -((bm[4 * k] + b0[4 * k]) + bp[4 * k]));
      y.y = fmaf(28.f, v0[4 * k + 1], -((bm[4 * k + 1] + b0[4 * k + 1]) + bp[4 * k + 1]));
      y.z = fmaf(28.f, v0[4 * k + 2], -((bm[4 * k + 2] + b0[4 * k + 2]) + bp[4 * k + 2]));
      y.w = fmaf(28.f, v0[4 * k + 3], -((bm[4 * k + 3] + b0[4 * k + 3]) + bp[4 * k + 3]));
      xv = make_float4(v0[4 * k], v0[4 * k + 1], v0[4 * k + 2], v0[4 * k + 3]);
      part += epi.store4(c0 + 4 * k + z * plane, y, xv);
    }
#pragma unroll
    for (int j = 0; j < W; ++j) {
      bm[j] = b0[j];
      b0[j] = bp[j];
      v0[j] = vp[j];
    }
  }
  return part;
}

// FP64 box walk, four columns per thread (map from boxw_map(4, ...)), for the
// outer residual of the refinement: the same reassociated sum as the FP32 box
// walk in double precision (not the reference's term order).
template <class Epi>
__device__ __forceinline__ double stencil_rows_box64x4(const StencilGeom &g, const PlaneMap &q,
                                                       const double *__restrict__ x, Epi &epi) {
  double part = 0.0;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)q.plane * q.nzc) return part;
  const int qz = (int)(t / q.plane);
  const int c0 = 4 * (int)(t - (int64_t)qz * q.plane);
  const int z0 = qz * q.zc, z1 = min(g.nz, z0 + q.zc);
  const int iy = c0 / g.nx, ix0 = c0 - iy * g.nx;
  const int plane = 4 * q.plane;
  const int dl = ix0 > 0 ? -1 : 0, dr = ix0 + 4 < g.nx ? 4 : 3;
  const double wl = ix0 > 0 ? 1.0 : 0.0, wr = ix0 + 4 < g.nx ? 1.0 : 0.0;
  const int ylo = iy > 0 ? -g.nx : 0, yhi = iy < g.ny - 1 ? g.nx : 0;
  const double wlo = iy > 0 ? 1.0 : 0.0, whi = iy < g.ny - 1 ? 1.0 : 0.0;
  const double *pc = x + c0;
  auto line = [&](const double *p, double *v, double *s) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
    const double l = wl * __ldg(p + dl), r = wr * __ldg(p + dr);
    s[0] = (l + v[0]) + v[1];
    s[1] = (v[0] + v[1]) + v[2];
    s[2] = (v[1] + v[2]) + v[3];
    s[3] = (v[2] + v[3]) + r;
  };
  auto box = [&](int z, double *bx, double *v) {
    const bool zin = (unsigned)z < (unsigned)g.nz;
    const double *p = pc + (int64_t)(zin ? z : 0) * plane;
    double s0[4], s1[4], s2[4], u[4];
    line(p + ylo, u, s0);
    line(p, v, s1);
    line(p + yhi, u, s2);
    const double wz = zin ? 1.0 : 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) bx[j] = wz * fma(wlo, s0[j], fma(whi, s2[j], s1[j]));
  };
  double bm[4], b0[4], bp[4], vm[4], v0[4], vp[4];
  box(z0 - 1, bm, vm);
  box(z0, b0, v0);
  for (int z = z0; z < z1; ++z) {
    box(z + 1, bp, vp);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      part += epi(c0 + j + z * plane, fma(28.0, v0[j], -((bm[j] + b0[j]) + bp[j])));
      bm[j] = b0[j];
      b0[j] = bp[j];
      v0[j] = vp[j];
    }
  }
  return part;
}

// The pipelined row sums of one column (the single-line form of ColumnPair2
// below): a row's 27 terms in the reference's order, split at the plane
// boundaries.  When plane p arrives, end() finishes the row of plane p-1 with
// p's nine values and middle() carries the row of plane p through its own
// plane and starts the nine-term prefix of the row of plane p+1 -- three
// independent 9-term chains a step instead of one 18-term chain.
template <typename Real>
struct ColumnLine {
  Real lead;  // the next plane's row: its first nine terms
  Real mid;   // the current plane's row: through its own plane
  Real x;     // x of the current plane's row
  __device__ __forceinline__ void first(const Real *v) { lead = stencil_lead<Real>(v); }
  __device__ __forceinline__ void middle(const Real *v) {
    mid = stencil_mid<Real>(lead, v);
    x = v[4];
    lead = stencil_lead<Real>(v);
  }
  __device__ __forceinline__ Real end(const Real *v) const { return stencil_end<Real>(mid, v); }
};

// The z walk of one column (plane map): planes z0-1 .. z1 of the column's 3x3
// neighbourhood, one plane a step.  epi(i, rowsum, x_i) stores and returns a
// dot term.
template <typename Real, class Epi>
__device__ __forceinline__ double stencil_column(const PlaneSpan &sp, const StencilGeom &g, const PlaneMap &m,
                                                 unsigned mask, const Real *__restrict__ pc, Epi &epi) {
  double part = 0.0;
  Real v[9];
  ColumnLine<Real> w;
  stencil_plane<Real>(pc + (int64_t)(sp.z0 - 1) * m.plane, g.nx, mask, sp.z0 > 0, v);
  w.first(v);
  stencil_plane<Real>(pc + (int64_t)sp.z0 * m.plane, g.nx, mask, true, v);
  w.middle(v);
  for (int z = sp.z0; z < sp.z1; ++z) {
    stencil_plane<Real>(pc + (int64_t)(z + 1) * m.plane, g.nx, mask, z + 1 < g.nz, v);
    const Real s = w.end(v);
    if constexpr (sizeof(Real) == 8)
      part = __dadd_rn(part, epi(sp.c + z * m.plane, s, w.x));
    else
      part += epi(sp.c + z * m.plane, s, w.x);
    w.middle(v);
  }
  return part;
}

// The 3x3 neighbourhood of an interior column in the plane `p` points into:
// three row pointers with +-1 offsets (immediates), no tests.
template <typename Real>
__device__ __forceinline__ void stencil_plane3(const Real *__restrict__ p, int nx, Real *v) {
  const Real *r0 = p - nx, *r2 = p + nx;
  v[0] = __ldg(r0 - 1), v[1] = __ldg(r0), v[2] = __ldg(r0 + 1);
  v[3] = __ldg(p - 1), v[4] = __ldg(p), v[5] = __ldg(p + 1);
  v[6] = __ldg(r2 - 1), v[7] = __ldg(r2), v[8] = __ldg(r2 + 1);
}
// stencil_column for a column whose nine neighbours lie inside the grid in x
// and y: the planes inside the grid load without selects (the plane above the
// grid's last one is zeros).  Same sums.
template <typename Real, class Epi>
__device__ __forceinline__ double stencil_column_interior(const PlaneSpan &sp, const StencilGeom &g,
                                                          const PlaneMap &m, const Real *__restrict__ pc,
                                                          Epi &epi) {
  double part = 0.0;
  Real v[9];
  ColumnLine<Real> w;
  const int64_t pl = m.plane;
  if (sp.z0 > 0) {
    stencil_plane3<Real>(pc + (sp.z0 - 1) * pl, g.nx, v);
  } else {
#pragma unroll
    for (int j = 0; j < 9; ++j) v[j] = Real(0);
  }
  w.first(v);
  stencil_plane3<Real>(pc + sp.z0 * pl, g.nx, v);
  w.middle(v);
  const int zi = min(sp.z1, g.nz - 1);  // rows whose plane z+1 lies inside the grid
  const Real *p = pc + (sp.z0 + 1) * pl;
  int z = sp.z0;
  for (; z < zi; ++z, p += pl) {
    stencil_plane3<Real>(p, g.nx, v);
    const Real s = w.end(v);
    if constexpr (sizeof(Real) == 8)
      part = __dadd_rn(part, epi(sp.c + z * m.plane, s, w.x));
    else
      part += epi(sp.c + z * m.plane, s, w.x);
    w.middle(v);
  }
  if (z < sp.z1) {  // z = nz - 1: no plane above
#pragma unroll
    for (int j = 0; j < 9; ++j) v[j] = Real(0);
    const Real s = w.end(v);
    if constexpr (sizeof(Real) == 8)
      part = __dadd_rn(part, epi(sp.c + z * m.plane, s, w.x));
    else
      part += epi(sp.c + z * m.plane, s, w.x);
  }
  return part;
}

// Lines y-1 .. y+2 (three values each, x-1 .. x+1) of the plane `p` points
// into (p = &x[column + z*plane], the column at an even line y): v[3l + k] is
// line y-1+l, x-1+k.  `mask` bit 3l+k clear (or zin false) gives 0 there.
template <typename Real, bool FULL>
__device__ __forceinline__ void stencil_plane4(const Real *__restrict__ p, int nx, unsigned mask, bool zin,
                                               Real *v) {
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    const int off = (j / 3 - 1) * nx + (j % 3 - 1);
    v[j] = (zin && (FULL || ((mask >> j) & 1u))) ? __ldg(p + off) : Real(0);
  }
}
// Bit 3l+k set when line y-1+l, column x-1+k of the pair (x, y), (x, y+1) is
// inside the grid.
__device__ __forceinline__ unsigned stencil_mask4(const StencilGeom &g, int ix, int iy) {
  unsigned mask = 0;
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    const int yy = iy + j / 3 - 1, xx = ix + j % 3 - 1;
    if ((unsigned)yy < (unsigned)g.ny && (unsigned)xx < (unsigned)g.nx) mask |= 1u << j;
  }
  return mask;
}
// The z walk of a column pair (x, y) and (x, y+1): per plane twelve loads serve
// both rows (nine a row otherwise).  Each row's sum is the single-line walk's,
// term for term: plane z-1 (lead), plane z (mid), plane z+1 (end), lines in sy
// order; row y's lines are v[0..8], row y+1's v[3..11].  The three pieces are
// pipelined across planes (ColumnPair2): when plane z+1 arrives it ends the
// rows of plane z, takes the rows of plane z+1 through their mid and starts
// the leads of plane z+2 -- six independent 9-term chains a step instead of
// two 18-term ones, and one plane of values held instead of two.  Rows go to
// epi in the order (z, y), (z, y+1), z ascending -- the order thread_rows
// gives the ELL kernels.
template <typename Real>
struct ColumnPair2 {
  Real lead0, lead1;  // rows of the next plane: their first nine terms
  Real mid0, mid1;    // rows of the current plane: through their plane's terms
  Real x0, x1;        // x of the current plane's two rows
  // plane z-1 of the walk's first row
  __device__ __forceinline__ void first(const Real *v) {
    lead0 = stencil_lead<Real>(v);
    lead1 = stencil_lead<Real>(v + 3);
  }
  // plane p: the rows of plane p through their mid, the leads of plane p+1
  __device__ __forceinline__ void middle(const Real *v) {
    mid0 = stencil_mid<Real>(lead0, v);
    mid1 = stencil_mid<Real>(lead1, v + 3);
    x0 = v[4];
    x1 = v[7];
    lead0 = stencil_lead<Real>(v);
    lead1 = stencil_lead<Real>(v + 3);
  }
  // plane p+1 ends the rows of plane p: s0, s1 (then middle(v) moves on)
  __device__ __forceinline__ void end(const Real *v, Real &s0, Real &s1) const {
    s0 = stencil_end<Real>(mid0, v);
    s1 = stencil_end<Real>(mid1, v + 3);
  }
};
template <typename Real, bool FULL, class Epi>
__device__ __forceinline__ double stencil_column2(const PlaneSpan &sp, const StencilGeom &g, const PlaneMap &m,
                                                  unsigned mask, const Real *__restrict__ pc, Epi &epi) {
  double part = 0.0;
  Real v[12];
  ColumnPair2<Real> w;
  stencil_plane4<Real, FULL>(pc + (int64_t)(sp.z0 - 1) * m.plane, g.nx, mask, sp.z0 > 0, v);
  w.first(v);
  stencil_plane4<Real, FULL>(pc + (int64_t)sp.z0 * m.plane, g.nx, mask, true, v);
  w.middle(v);
  for (int z = sp.z0; z < sp.z1; ++z) {
    stencil_plane4<Real, FULL>(pc + (int64_t)(z + 1) * m.plane, g.nx, mask, z + 1 < g.nz, v);
    Real s0, s1;
    w.end(v, s0, s1);
    if constexpr (sizeof(Real) == 8) {
      part = __dadd_rn(part, epi(sp.c + z * m.plane, s0, w.x0));
      part = __dadd_rn(part, epi(sp.c + g.nx + z * m.plane, s1, w.x1));
    } else {
      part += epi(sp.c + z * m.plane, s0, w.x0);
      part += epi(sp.c + g.nx + z * m.plane, s1, w.x1);
    }
    w.middle(v);
  }
  return part;
}

// All rows of the calling thread; epi(i, rowsum, x_i) stores and returns a dot term.
template <typename Real, class Epi>
__device__ __forceinline__ double stencil_rows(int n, const StencilGeom &g, const PlaneMap &m,
                                               const Real *__restrict__ x, Epi &epi) {
  double part = 0.0;
  if (m.plane > 0) {
    PlaneSpan sp;
    if (m.tiles_x > 0) {
      const TileSpan ts = tile_span(m, g.nz);
      if (!ts.rows) return part;
      sp = PlaneSpan{ts.c, ts.z0, ts.z1};
    } else {
      sp = plane_span(m, g.nz);
    }
    if (sp.z0 >= sp.z1) return part;
    const int iy = sp.c / g.nx, ix = sp.c - iy * g.nx;
    if (m.ry == 2) {
      const unsigned mask4 = stencil_mask4(g, ix, iy);
      if (__all_sync(__activemask(), mask4 == 0xFFFu))
        return stencil_column2<Real, true>(sp, g, m, mask4, x + sp.c, epi);
      return stencil_column2<Real, false>(sp, g, m, mask4, x + sp.c, epi);
    }
    const unsigned mask = stencil_mask(g, ix, iy);
    // warps whose columns all lie off the x and y faces load without the
    // per-neighbour tests (the sums are the same: masked terms are zeros)
    if (__all_sync(__activemask(), mask == 0x1FFu))
      return stencil_column_interior<Real>(sp, g, m, x + sp.c, epi);
    return stencil_column<Real>(sp, g, m, mask, x + sp.c, epi);
  }
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const Real s = stencil_row<Real>(i, g, x);
    if constexpr (sizeof(Real) == 8)
      part = __dadd_rn(part, epi(i, s));
    else
      part += epi(i, s);
  }
  return part;
}

}  // namespace hpccg
