// unet_conv.cuh -- 3x3x3 convolutions with 16 output channels on tcgen05.
//
// Activation layout ("row-planar"): a 16-channel tensor of nb grids of
// nx*ny*nz voxels is stored as [b][z][y][h][x][8] -- for every grid row
// (b,z,y), first the 8-channel half h=0 of all nx voxels, then h=1.  A voxel
// half is one 16-byte unit, and a run of consecutive voxels of one row and
// half is one contiguous span, which is exactly the layout the tensor cores
// read (no-swizzle K-major core matrices: 8 rows x 16 bytes; the two halves
// are the two K chunks).  So every operand tile arrives by 1D bulk copies
// (cp.async.bulk) of whole row spans, with zero fill at the grid faces.
//
// A conv is an implicit GEMM per tile of 128 (or 64) voxels: for each of the
// 27 taps and each 16-channel input group, one tcgen05.mma (M=128 or 64,
// N=16, K=16) accumulates into a 16-column FP32 TMEM accumulator.
//  * row tiles (nx a multiple of 128, or nx = 64 with M = 64): a tile is one
//    x-row; the 3x3 neighbouring rows with a 1-voxel x halo are three "slabs"
//    shared with the neighbouring tiles in y, and the 27 taps read them through
//    shifted descriptors (one new slab fetched per tile);
//  * brick tiles (other narrow grids): a tile is a bx*by*bz brick of 128
//    voxels and each tap's shifted brick is fetched separately.
// Roles per pipeline (192 threads): warp 0 fetches (its lanes issue the row
// spans in parallel), warp 1 allocates TMEM and lane 0 issues the MMAs, warps
// 2-5 (one per TMEM lane quarter) run the epilogue.  Row kernels of 32-channel
// layers run two such pipelines per CTA (384 threads) that share the weights.
#pragma once
#include "hpccg_internal.cuh"
#include "unet_tc.cuh"

namespace hpccg {

// Offsets in the row-planar layout; row = (b*nz + z)*ny + y.
__host__ __device__ __forceinline__ int64_t act_unit(int64_t row, int h, int x, int nx) {
  return (row * 2 + h) * (int64_t)nx + x;
}
__host__ __device__ __forceinline__ int64_t act_elem(int64_t row, int x, int c, int nx) {
  return act_unit(row, c >> 3, x, nx) * 8 + (c & 7);
}

constexpr int kConvThreads = 192;
constexpr int kWTapBytes = 16 * 16 * 2;  // one tap of B: 16 x 16 BF16

// Brick tiles: one stage per k-step (tap, input): 2 halves x 128 units.
constexpr int kBrickStages = 24;
constexpr int kBrickStageBytes = 2 * 128 * 16;
// Row tiles of RX = 128 voxels (nx a multiple of 128; MMA M = 128) or RX = 64
// (nx = 64; M = 64) walk y inside a work unit (b, z, RX-voxel x block, chunk of
// up to row_chunk(RX) rows of y).  A "slab" is grid row y of the three z planes
// z-1, z, z+1 with a 1-voxel x halo: 3 rows x (RX + 2) units per half.  Tile y
// reads slabs y-1, y, y+1, so each tile fetches one new slab and a ring of
// row_slots slabs keeps several fetches in flight.
__host__ __device__ constexpr int row_vox(int rx) { return rx + 2; }
__host__ __device__ constexpr int row_chunk(int rx) { return rx == 128 ? 32 : 8; }
__host__ __device__ constexpr int slab_plane_bytes(int rx) { return ((3 * row_vox(rx) * 16 + 127) / 128) * 128; }
__host__ __device__ constexpr int slab_bytes(int nin, int rx) { return nin * 2 * slab_plane_bytes(rx); }
__host__ __device__ constexpr int row_slots(int nin, int rx, int pipes = 1) {
  return pipes == 2 ? 4 : ((rx == 128 && nin == 1) ? 8 : 6);
}
// Row kernels may run two independent pipelines (producer, MMA issuer and
// epilogue warps each, own slab ring and accumulators) in one CTA that shares
// the weights: two MMA-issuing threads per SM where the shared memory of one
// pipeline per CTA leaves room for only one CTA.
__host__ __device__ constexpr int row_pipes(int nin, int rx) { return (nin == 2 && rx == 128) ? 2 : 1; }
// mbarriers: full[S], empty[S], acc_full[2], acc_empty[2], drain, + TMEM slot.
__host__ __device__ constexpr int bar_bytes(int stages) { return (2 * stages + 5) * 8 + 16; }
__host__ __device__ constexpr int brick_smem_bytes(int nin) {
  return nin * 27 * kWTapBytes + kBrickStages * kBrickStageBytes + bar_bytes(kBrickStages);
}
// One pipeline's ring and barriers, rounded up so that the next ring starts on
// a 128-byte boundary (bulk copies and MMA operands need 16-byte alignment).
__host__ __device__ constexpr int row_pipe_bytes(int nin, int rx) {
  return ((row_slots(nin, rx, row_pipes(nin, rx)) * slab_bytes(nin, rx) +
           bar_bytes(row_slots(nin, rx, row_pipes(nin, rx))) + 127) / 128) * 128;
}
__host__ __device__ constexpr int row_smem_bytes(int nin, int rx) {
  return nin * 27 * kWTapBytes + row_pipes(nin, rx) * row_pipe_bytes(nin, rx);
}

enum ConvEpi : int {
  kEpiBiasRelu = 0,   // out_bf16 = relu(acc + bias)
  kEpiBias = 1,       // out_bf16 = acc + bias
  kEpiProject = 2,    // out_f32[voxel] = proj . relu(acc + bias) + proj_bias
  kEpiRawF32 = 3,     // out_f32 = acc (16 channels, row-planar)
};

struct ConvGeom {
  int nx, ny, nz, nb;  // volume and batch
  int bx, by, bz;      // tile brick (bx*by*bz = 128)
  int tx, ty, tz;      // tiles per dimension
  int ntiles;
};

struct ConvArgs {
  ConvGeom g;
  const __nv_bfloat16 *in0, *in1;  // row-planar inputs
  const __nv_bfloat16 *wpack;      // [nin][27][2][16][8] BF16
  const float *bias;               // [16] (null for kEpiRawF32)
  const float *proj;               // [17] for kEpiProject
  void *out;
  int *err;
};

// Host: brick and tile counts for a volume (dims must be divisible by the brick).
inline bool conv_geom(int nx, int ny, int nz, int nb, ConvGeom *g) {
  if ((int64_t)nx * ny * nz < 128) return false;
  int bx = nx < 128 ? nx : 128;
  int by = 128 / bx;
  if (by > ny) by = ny;
  int bz = 128 / (bx * by);
  if (bx < 8 || bx * by * bz != 128 || nx % bx || ny % by || nz % bz) return false;
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  g->nb = nb;
  g->bx = bx;
  g->by = by;
  g->bz = bz;
  g->tx = nx / bx;
  g->ty = ny / by;
  g->tz = nz / bz;
  g->ntiles = g->tx * g->ty * g->tz * nb;
  return true;
}
inline bool conv_row_ok(const ConvGeom &g) { return g.bx == 128 && g.by == 1 && g.bz == 1; }
// Geometry of 64-voxel row tiles for nx = 64 (tile = one grid row).
inline bool conv_row64_geom(const ConvGeom &g, ConvGeom *r) {
  if (g.nx != 64) return false;
  *r = g;
  r->bx = 64;
  r->by = 1;
  r->bz = 1;
  r->tx = 1;
  r->ty = g.ny;
  r->tz = g.nz;
  r->ntiles = g.ny * g.nz * g.nb;
  return true;
}

// Launches the tensor-core conv (row tiles when possible unless force_brick).
int launch_conv3_tc(int nin, int epi, const ConvArgs &a, int num_sms, cudaStream_t s, bool force_brick = false);
// The 1-channel input layer (FP32 input [nb][nz][ny][nx], W [27][16], bias [16])
// on the tensor cores, BF16 operands, FP32 accumulation; nx a multiple of 128,
// else HPCCG_ERR_UNSUPPORTED.
int launch_conv3_in1_tc(const float *in, const float *W, const float *bias, __nv_bfloat16 *out, int nx, int ny,
                        int nz, int nb, int relu, int *err, int num_sms, cudaStream_t s);

}  // namespace hpccg
