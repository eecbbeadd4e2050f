// hpccg_stencil_tma64.cuh -- FP64 matrix-free walks of the generate_matrix
// operator (MPI/src/SparseMatrix.F90:138-159, spmv :213-232) with their input
// streamed by TMA.
//
// A CTA owns a rectangle of grid columns and a chunk of z planes.  Thread 0
// issues one 3D tensor load per plane (the rectangle with a one-wide halo in
// y and a two-wide one in x, so that the x start stays on a 16-byte boundary)
// into a ring of shared-memory slots, several planes ahead of the plane being
// read; planes and columns outside the grid arrive as +0.0 (tensor-map
// out-of-bounds fill), so the sums need no masks.
//
//  * stencil_rows_tma64box: 32 x 64 columns per CTA, 4 x 2 columns a thread,
//    the reassociated FP64 sum of stencil_rows_box64x4 (3-point line sums, 3x3
//    box sums, y = 28 x - (box(z-1) + box(z) + box(z+1))), the same value bit
//    for bit up to the sign of a zero.  The refinement residual of the mixed
//    solvers; b arrives by TMA in the same slots.
//  * stencil_rows_tma64ref: 32 x 16 columns per CTA, the column pair (x, y),
//    (x, y+1) of an even line y a thread, the reference's term order
//    (stencil_column2), so the row sums are bit-identical to the ELL kernels'.
//    The rows of a thread and their order are those of thread_rows under the
//    same tile map, so fused dots -- and whole CG runs -- are bit-identical
//    between the two.
//
// Waits on the ring's mbarriers are bounded: on expiry the CTA records
// HPCCG_ERR_TIMEOUT in the caller's status word, waits (bounded) for its own
// loads in flight and finishes without the remaining rows.
#pragma once
#include "hpccg_stencil.cuh"
#include "hpccg_stencil_tma.cuh"

namespace hpccg {

// Host: the tensor map of a FP64 grid vector x[nz][ny][nx] (base 16-byte
// aligned, nx even), box box_x x box_y x 1.
int make_stencil_tmap64(CUtensorMap *map, const double *base, int nx, int ny, int nz, int box_x, int box_y);

// A ring of STAGES shared-memory slots, each receiving one z plane of the
// CTA's box.  Planes lo .. hi load in order; thread 0 issues them, STAGES
// ahead of the plane being read.
// A slot can also take a companion box: plane p + 1 of map2 for p + 1 in
// [lo2, hi2], at byte offset off2 of the slot (the same mbarrier covers both).
template <int STAGES>
struct PlaneRing {
  unsigned char *slots;
  int slot_bytes;
  uint64_t *full;  // [STAGES] mbarriers in shared memory
  const CUtensorMap *map;
  int bx, by;      // box origin (x, y)
  uint32_t bytes;  // bytes one plane delivers
  int lo, hi;
  int next;      // thread 0: the next plane to issue
  int consumed;  // the last plane every thread has released
  const CUtensorMap *map2 = nullptr;
  int bx2 = 0, by2 = 0, off2 = 0, lo2 = 0, hi2 = -1;
  uint32_t bytes2 = 0;

  __device__ __forceinline__ int slot(int p) const { return (p - lo) % STAGES; }
  __device__ __forceinline__ uint32_t parity(int p) const { return (uint32_t)((p - lo) / STAGES) & 1u; }
  __device__ __forceinline__ const unsigned char *data(int p) const { return slots + (size_t)slot(p) * slot_bytes; }
  __device__ __forceinline__ void issue() {  // thread 0
    const int k = slot(next);
    const bool two = map2 && next - 1 >= lo2 && next - 1 <= hi2;
    tc::mbar_expect_tx(&full[k], bytes + (two ? bytes2 : 0u));
    tma_load_3d(slots + (size_t)k * slot_bytes, map, &full[k], bx, by, next);
    if (two) tma_load_3d(slots + (size_t)k * slot_bytes + off2, map2, &full[k], bx2, by2, next - 1);
    ++next;
  }
  // Thread 0 initialises the barriers; a CTA barrier must follow, then prime().
  __device__ __forceinline__ void init() {
    next = lo;
    consumed = lo - 1;
    if (threadIdx.x == 0) {
      for (int k = 0; k < STAGES; ++k) tc::mbar_init(&full[k], 1);
      tc::fence_mbar_init();
    }
  }
  __device__ __forceinline__ void prime() {
    if (threadIdx.x == 0)
      while (next <= hi && next < lo + STAGES) issue();
  }
  // Bounded wait until plane p has landed; false on expiry (recorded in status).
  __device__ __forceinline__ bool wait(int p, int *status) const {
    for (uint32_t i = 0;; ++i) {
      if (tc::mbar_try_wait(&full[slot(p)], parity(p))) return true;
      if (i >= tc::kSpinLimit) {
        if (status) atomicCAS(status, 0, HPCCG_ERR_TIMEOUT);
        return false;
      }
    }
  }
  // CTA barrier once every thread has read plane p; its slot then takes the
  // next plane.  False in every thread when any thread's wait expired.
  __device__ __forceinline__ bool release(int p, bool ok) {
    if (__syncthreads_or(!ok)) return false;
    consumed = p;
    if (threadIdx.x == 0 && next <= hi) issue();
    return true;
  }
  // Thread 0, after a failure: the loads still in flight land before the CTA exits.
  __device__ __forceinline__ void drain() const {
    if (threadIdx.x != 0) return;
    for (int p = consumed + 1; p < next; ++p)
      for (uint32_t i = 0; i < tc::kSpinLimit; ++i)
        if (tc::mbar_try_wait(&full[slot(p)], parity(p))) break;
  }
};

// ---- reassociated FP64 box walk (refinement residual) -----------------------
constexpr int kB64TileX = 32, kB64TileY = 64;                  // columns per CTA
constexpr int kB64BoxX = kB64TileX + 4;                        // x0-2 .. x0+33
constexpr int kB64BoxY = kB64TileY + 2;                        // y0-1 .. y0+64
constexpr uint32_t kB64BoxBytes = kB64BoxX * kB64BoxY * 8;     // 19008
constexpr int kB64XSlot = ((kB64BoxBytes + 127) / 128) * 128;  // 19072
constexpr uint32_t kB64TileBytes = kB64TileX * kB64TileY * 8;   // 16384: the companion tile (b)
constexpr int kB64Slot = kB64XSlot + kB64TileBytes;             // 35456
constexpr int kB64Stages = 3;
constexpr int kB64RingBytes = kB64Stages * kB64Slot;           // dynamic shared memory (two CTAs a SM)
static_assert(kBlock == (kB64TileX / 4) * (kB64TileY / 2), "one thread per 4 x 2 columns");

// Rows of the calling CTA (tile plan with kB64TileX x kB64TileY tiles).  With
// the slot of plane z+1 arrives the tile of plane z of a second vector (bmap,
// no halo); epi.store4(i, y[4], b4) stores rows i .. i+3 and returns their
// dot term, b4 = that vector's four values of the rows (shared memory).
// Every thread of the CTA must call it (it has barriers).
template <class Epi>
__device__ __forceinline__ double stencil_rows_tma64box(const TmaTile &t, const CUtensorMap *map,
                                                        const CUtensorMap *bmap, Epi &epi, int *status) {
  extern __shared__ __align__(128) unsigned char b64_ring[];  // kB64RingBytes
  __shared__ uint64_t full[kB64Stages];
  double part = 0.0;
  const int tid = threadIdx.x, tx = tid & 7, ty = tid >> 3;
  const int per_plane = t.tiles_x * t.tiles_y;
  const int q = blockIdx.x / per_plane, tile = blockIdx.x - q * per_plane;
  const int x0 = (tile % t.tiles_x) * kB64TileX, y0 = (tile / t.tiles_x) * kB64TileY;
  const int z0 = q * t.zc, z1 = min(t.nz, z0 + t.zc);
  const int xc = x0 + 4 * tx, yc = y0 + 2 * ty;
  const int64_t plane = (int64_t)t.nx * t.ny;
  PlaneRing<kB64Stages> ring{b64_ring, kB64Slot, full, map, x0 - 2, y0 - 1, kB64BoxBytes, z0 - 1, z1, 0, 0};
  ring.map2 = bmap;  // b(z) rides with x(z+1), z in [z0, z1)
  ring.bx2 = x0;
  ring.by2 = y0;
  ring.off2 = kB64XSlot;
  ring.bytes2 = kB64TileBytes;
  ring.lo2 = z0;
  ring.hi2 = z1 - 1;
  ring.init();
  __syncthreads();
  ring.prime();
  // box sums (b) and centres (v) of plane p for the thread's 4 x 2 columns:
  // line sums (l + v0) + v1, (v0 + v1) + v2, ...; box = s(y-1) + (s(y+1) + s(y))
  auto consume = [&](int p, double (*b)[4], double (*v)[4]) -> bool {
    if (!ring.wait(p, status)) return false;
    const double *c = reinterpret_cast<const double *>(ring.data(p)) + (2 * ty) * kB64BoxX + 2 + 4 * tx;
    double ls[4][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double *r = c + k * kB64BoxX;
      const double2 a = *reinterpret_cast<const double2 *>(r);
      const double2 e = *reinterpret_cast<const double2 *>(r + 2);
      const double l = r[-1], rr = r[4];
      if (k == 1 || k == 2) {
        v[k - 1][0] = a.x, v[k - 1][1] = a.y, v[k - 1][2] = e.x, v[k - 1][3] = e.y;
      }
      ls[k][0] = (l + a.x) + a.y;
      ls[k][1] = (a.x + a.y) + e.x;
      ls[k][2] = (a.y + e.x) + e.y;
      ls[k][3] = (e.x + e.y) + rr;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 4; ++i) b[j][i] = ls[j][i] + (ls[j + 2][i] + ls[j + 1][i]);
    return true;
  };
  double bm[2][4], b0[2][4], bp[2][4], vm[2][4], v0[2][4], vp[2][4];
  bool ok = consume(z0 - 1, bm, vm);
  if (ring.release(z0 - 1, ok)) {
    ok = consume(z0, b0, v0);
    if (ring.release(z0, ok)) {
      for (int z = z0; z < z1; ++z) {
        ok = consume(z + 1, bp, vp);
        if (ok) {  // rows of plane z, before the slot that holds b(z) is released
          const double *bt = reinterpret_cast<const double *>(ring.data(z + 1) + kB64XSlot) +
                             (2 * ty) * kB64TileX + 4 * tx;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            if (xc < t.nx && yc + j < t.ny) {
              double y[4];
#pragma unroll
              for (int i = 0; i < 4; ++i) y[i] = fma(28.0, v0[j][i], -((bm[j][i] + b0[j][i]) + bp[j][i]));
              part = __dadd_rn(part, epi.store4((int)(z * plane + (int64_t)(yc + j) * t.nx + xc), y,
                                                bt + j * kB64TileX));
            }
          }
        }
        if (!ring.release(z + 1, ok)) break;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            bm[j][i] = b0[j][i];
            b0[j][i] = bp[j][i];
            v0[j][i] = vp[j][i];
          }
      }
    }
  }
  if (ring.consumed < z1) ring.drain();
  return part;
}

// ---- reference-order FP64 walk (CG SpMV) --------------------------------------
constexpr int kR64TileX = kTileX, kR64TileY = kTileY;                 // 32 x 16 columns per CTA
constexpr int kR64BoxX = kR64TileX + 4;                               // x0-2 .. x0+33
constexpr int kR64BoxY = kR64TileY + 2;                               // y0-1 .. y0+16
constexpr uint32_t kR64BoxBytes = kR64BoxX * kR64BoxY * 8;            // 5184
constexpr int kR64Slot = ((kR64BoxBytes + 127) / 128) * 128;          // 5248
constexpr int kR64Stages = 6;
constexpr int kR64RingBytes = kR64Stages * kR64Slot;                  // 31488, static shared memory

// Rows of the calling CTA under the tile map m (m.tiles_x > 0); epi(i, rowsum,
// x_i) stores and returns a dot term, rows (z, y) then (z, y+1), z ascending.
// Every thread of the CTA must call it (it has barriers).
template <class Epi>
__device__ __forceinline__ double stencil_rows_tma64ref(const StencilGeom &g, const PlaneMap &m,
                                                        const CUtensorMap *map, Epi &epi, int *status) {
  __shared__ __align__(128) unsigned char r64_ring[kR64RingBytes];
  __shared__ uint64_t full[kR64Stages];
  double part = 0.0;
  const TileSpan sp = tile_span(m, g.nz);
  PlaneRing<kR64Stages> ring{r64_ring, kR64Slot, full, map, sp.x0 - 2, sp.y0 - 1, kR64BoxBytes, sp.z0 - 1, sp.z1,
                             0, 0};
  ring.init();
  __syncthreads();
  ring.prime();
  const int tx = threadIdx.x % kR64TileX, ty = threadIdx.x / kR64TileX;
  const int ofs = (2 * ty) * kR64BoxX + 1 + tx;  // box position of (x-1, y-1)
  // lines y-1 .. y+2 of plane p, columns x-1 .. x+1: v[3l + k]
  auto consume = [&](int p, double *v) -> bool {
    if (!ring.wait(p, status)) return false;
    const double *c = reinterpret_cast<const double *>(ring.data(p)) + ofs;
#pragma unroll
    for (int j = 0; j < 12; ++j) v[j] = c[(j / 3) * kR64BoxX + j % 3];
    return true;
  };
  double v[12];
  ColumnPair2<double> w;  // the pipelined sums of stencil_column2
  bool ok = consume(sp.z0 - 1, v);
  w.first(v);
  if (ring.release(sp.z0 - 1, ok)) {
    ok = consume(sp.z0, v);
    w.middle(v);
    if (ring.release(sp.z0, ok)) {
      for (int z = sp.z0; z < sp.z1; ++z) {
        ok = consume(z + 1, v);
        if (!ring.release(z + 1, ok)) break;
        double s0, s1;
        w.end(v, s0, s1);
        if (sp.rows) {
          part = __dadd_rn(part, epi(sp.c + z * m.plane, s0, w.x0));
          part = __dadd_rn(part, epi(sp.c + g.nx + z * m.plane, s1, w.x1));
        }
        w.middle(v);
      }
    }
  }
  if (ring.consumed < sp.z1) ring.drain();
  return part;
}

}  // namespace hpccg
