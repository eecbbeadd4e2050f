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
// bit-identical to the CSR/ELL kernels'.  Rows map to threads exactly as in
// ell_rows<..., RPT=1> (thread t: rows t, t+stride, ...), so fused dot
// products, and with them whole CG runs, are bit-identical too.
#pragma once
#include "hpccg_internal.cuh"

namespace hpccg {

struct StencilGeom {
  int nx, ny, nz;
};

template <typename Real>
__device__ __forceinline__ Real stencil_row(int i, const StencilGeom &g, const Real *__restrict__ x) {
  const int nxy = g.nx * g.ny;
  const int iz = i / nxy, rem = i - iz * nxy;
  const int iy = rem / g.nx, ix = rem - iy * g.nx;
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

// Grid-stride walk over the rows; epi(i, rowsum) stores and returns a dot term.
template <typename Real, class Epi>
__device__ __forceinline__ double stencil_rows(int n, const StencilGeom &g, const Real *__restrict__ x,
                                               Epi &epi) {
  double part = 0.0;
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
