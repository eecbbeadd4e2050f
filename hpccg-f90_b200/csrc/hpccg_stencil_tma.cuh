// hpccg_stencil_tma.cuh -- the FP32 matrix-free SpMV of the inner solves with
// its input streamed by TMA: a CTA owns a 32 x 64 tile of grid columns and a
// chunk of z planes; one thread issues 3D tensor loads of the tile with its
// halo (40 x 66 floats, the x start rounded down to a 16-byte boundary) into a
// ring of kTmaStages shared-memory slots, kTmaStages planes ahead of the row
// being summed.  Planes and rows outside the grid arrive as zeros (tensor-map
// out-of-bounds fill), so the sums need no masks.  Each thread forms the 3x3
// box sums of its 4 x 2 columns from shared memory (4 grid lines serve both rows), keeps three planes of box sums
// in registers and writes y_i = 28 x_i - (box(z-1) + box(z) + box(z+1)), the
// same reassociated FP32 sum as stencil_rows_boxw.
//
// Waits on the ring's mbarriers are bounded: on expiry the CTA records
// HPCCG_ERR_TIMEOUT in the caller's status word, waits (bounded) for its own
// loads in flight and finishes without the remaining rows.
#pragma once
#include <cuda.h>

#include "hpccg_internal.cuh"
#include "unet_tc.cuh"

namespace hpccg {

constexpr int kTmaRows = 2;                             // grid rows (y) per thread
constexpr int kTmaTileX = 32, kTmaTileY = 32 * kTmaRows;  // columns per CTA
constexpr int kTmaBoxX = kTmaTileX + 8;                 // x0-4 .. x0+35 (16-byte aligned start)
constexpr int kTmaBoxY = kTmaTileY + 2;                 // y0-1 .. y0+TY
constexpr int kTmaSlotFloats = ((kTmaBoxX * kTmaBoxY * 4 + 127) / 128) * 128 / 4;
constexpr int kTmaStages = 6;
constexpr int kTmaRingBytes = kTmaStages * kTmaSlotFloats * 4;  // dynamic shared memory of the kernels
constexpr uint32_t kTmaBoxBytes = kTmaBoxX * kTmaBoxY * 4;
static_assert(kBlock == (kTmaTileX / 4) * (kTmaTileY / kTmaRows), "one thread per 4 x kTmaRows columns");

struct TmaTile {
  int nx, ny, nz;
  int tiles_x, tiles_y;  // tiles per plane
  int zc, nzc;           // z planes per CTA, z chunks
};

// Host: tiles and z chunks for one wave of `resident_ctas` CTAs; nzc = 0 when
// the grid does not allow the tensor map (nx not a multiple of 4).
inline TmaTile tma_tile_plan(int nx, int ny, int nz, int resident_ctas, int tile_x = kTmaTileX,
                             int tile_y = kTmaTileY) {
  TmaTile t{nx, ny, nz, 0, 0, 0, 0};
  if (nx < 4 || ny < 1 || nz < 1 || nx % 4) return t;
  t.tiles_x = (nx + tile_x - 1) / tile_x;
  t.tiles_y = (ny + tile_y - 1) / tile_y;
  const int per_plane = t.tiles_x * t.tiles_y;
  int k = resident_ctas / per_plane;
  k = k < 1 ? 1 : (k > nz ? nz : k);
  t.zc = (nz + k - 1) / k;
  t.nzc = (nz + t.zc - 1) / t.zc;
  if ((int64_t)per_plane * t.nzc > kMaxPartials) t.nzc = 0;  // keep the reduction scratch
  return t;
}
inline int tma_tile_grid(const TmaTile &t) { return t.tiles_x * t.tiles_y * t.nzc; }

// Host: the tensor map of a FP32 grid vector x[nz][ny][nx] (base 16-byte aligned),
// box box_x x box_y x 1.
int make_stencil_tmap(CUtensorMap *map, const float *base, int nx, int ny, int nz, int box_y = kTmaBoxY,
                      int box_x = kTmaBoxX);

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(tc::smem_u32(bar))
      : "memory");
}

// Rows of the calling CTA; epi.store4(i, y, x) stores four rows and returns
// their dot term.  Every thread of the CTA must call it (it has barriers).
template <class Epi>
__device__ __forceinline__ double stencil_rows_tma(const TmaTile &t, const CUtensorMap *map, Epi &epi,
                                                   int *status) {
  extern __shared__ __align__(128) unsigned char tma_ring[];  // kTmaRingBytes
  float *ring = reinterpret_cast<float *>(tma_ring);
  __shared__ uint64_t full[kTmaStages];
  __shared__ int s_fail;
  double part = 0.0;
  const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
  const int per_plane = t.tiles_x * t.tiles_y;
  const int q = blockIdx.x / per_plane, tile = blockIdx.x - q * per_plane;
  const int x0 = (tile % t.tiles_x) * kTmaTileX, y0 = (tile / t.tiles_x) * kTmaTileY;
  const int z0 = q * t.zc, z1 = min(t.nz, z0 + t.zc);
  const int xc = x0 + 4 * tx, yc = y0 + kTmaRows * ty;  // rows yc .. yc + kTmaRows - 1
  const int64_t plane = (int64_t)t.nx * t.ny;
  if (tid == 0) {
    for (int s = 0; s < kTmaStages; ++s) tc::mbar_init(&full[s], 1);
    tc::fence_mbar_init();
    s_fail = 0;
  }
  __syncthreads();
  // plane p lives in slot (p - (z0-1)) % S; its n-th use of that slot has parity n & 1
  auto slot_of = [&](int p) { return (p - z0 + 1) % kTmaStages; };
  auto issue = [&](int p) {  // thread 0
    const int s = slot_of(p);
    tc::mbar_expect_tx(&full[s], kTmaBoxBytes);
    tma_load_3d(ring + s * kTmaSlotFloats, map, &full[s], x0 - 4, y0 - 1, p);
  };
  int next = z0 - 1;  // next plane to load (thread 0's view)
  if (tid == 0)
    for (; next <= z1 && next < z0 - 1 + kTmaStages; ++next) issue(next);
  // box sums (and centres) of plane p for this thread's 4 x kTmaRows columns
  auto consume = [&](int p, float (*b)[4], float4 *v) -> bool {
    const int s = slot_of(p);
    const uint32_t parity = (uint32_t)((p - z0 + 1) / kTmaStages) & 1u;
    bool ok = true;
    for (uint32_t i = 0;; ++i) {
      if (tc::mbar_try_wait(&full[s], parity)) break;
      if (i >= tc::kSpinLimit) {
        ok = false;
        break;
      }
    }
    if (!ok) {
      s_fail = 1;
      if (status) atomicCAS(status, 0, HPCCG_ERR_TIMEOUT);
      return false;
    }
    // 3-point line sums of the kTmaRows + 2 grid lines yc-1 .. yc+kTmaRows (box rows kTmaRows*ty ..)
    const float *c = ring + s * kTmaSlotFloats + (kTmaRows * ty) * kTmaBoxX + 4 + 4 * tx;
    float ls[kTmaRows + 2][4];
#pragma unroll
    for (int k = 0; k < kTmaRows + 2; ++k) {
      const float *r = c + k * kTmaBoxX;
      const float4 m = *reinterpret_cast<const float4 *>(r);
      const float l = r[-1], rr = r[4];
      if (k >= 1 && k <= kTmaRows) v[k - 1] = m;
      ls[k][0] = (l + m.x) + m.y;
      ls[k][1] = (m.x + m.y) + m.z;
      ls[k][2] = (m.y + m.z) + m.w;
      ls[k][3] = (m.z + m.w) + rr;
    }
#pragma unroll
    for (int j = 0; j < kTmaRows; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) b[j][i] = (ls[j][i] + ls[j + 1][i]) + ls[j + 2][i];
    return true;
  };
  // after every thread has read plane p its slot takes plane p + S
  auto release = [&]() -> bool {
    __syncthreads();
    const bool failed = s_fail != 0;
    if (!failed && tid == 0 && next <= z1) {
      issue(next);
      ++next;
    }
    return !failed;
  };
  float bm[kTmaRows][4], b0[kTmaRows][4], bp[kTmaRows][4];
  float4 vm[kTmaRows], v0[kTmaRows], vp[kTmaRows];
  int consumed = z0 - 2;  // last plane consumed by every thread
  bool ok = consume(z0 - 1, bm, vm);
  if (release() && ok) {
    consumed = z0 - 1;
    ok = consume(z0, b0, v0);
    if (release() && ok) {
      consumed = z0;
      for (int z = z0; z < z1; ++z) {
        ok = consume(z + 1, bp, vp);
        if (!release() || !ok) break;
        consumed = z + 1;
#pragma unroll
        for (int j = 0; j < kTmaRows; ++j) {
          if (xc < t.nx && yc + j < t.ny) {
            float4 y;
            y.x = fmaf(28.f, v0[j].x, -((bm[j][0] + b0[j][0]) + bp[j][0]));
            y.y = fmaf(28.f, v0[j].y, -((bm[j][1] + b0[j][1]) + bp[j][1]));
            y.z = fmaf(28.f, v0[j].z, -((bm[j][2] + b0[j][2]) + bp[j][2]));
            y.w = fmaf(28.f, v0[j].w, -((bm[j][3] + b0[j][3]) + bp[j][3]));
            part += epi.store4((int)(z * plane + (int64_t)(yc + j) * t.nx + xc), y, v0[j]);
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            bm[j][i] = b0[j][i];
            b0[j][i] = bp[j][i];
          }
          v0[j] = vp[j];
        }
      }
    }
  }
  if (s_fail && tid == 0) {  // loads still in flight land before the CTA exits
    for (int p = consumed + 1; p < next; ++p) {
      const int s = slot_of(p);
      const uint32_t parity = (uint32_t)((p - z0 + 1) / kTmaStages) & 1u;
      for (uint32_t i = 0; i < tc::kSpinLimit; ++i)
        if (tc::mbar_try_wait(&full[s], parity)) break;
    }
  }
  return part;
}

}  // namespace hpccg
