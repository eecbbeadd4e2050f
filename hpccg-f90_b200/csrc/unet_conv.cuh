// unet_conv.cuh -- 3x3x3 convolutions with 16 output channels on tcgen05.
//
// Layout: activations are channels-last BF16, [batch][z][y][x][16].  A conv
// is an implicit GEMM per tile of 128 voxels (a bx*by*bz brick, one TMEM lane
// per voxel): for each of the 27 taps and each 16-channel input, the shifted
// brick is fetched by TMA (zero fill outside the volume = zero padding) and
// one tcgen05.mma (M=128, N=16, K=16) accumulates it into a 16-column FP32
// TMEM accumulator.
//
// Roles per CTA (192 threads): warp 0 lane 0 issues TMA loads into an S-stage
// ring, warp 1 allocates TMEM and lane 0 issues the MMAs, warps 2-5 (one per
// TMEM lane quarter) run the epilogue.  Two accumulators let the epilogue of
// one tile overlap the MMAs of the next.
//
// Shared-memory operands use the no-swizzle K-major core-matrix layout: A is
// [k-chunk 2][voxel 128][8 channels] (two TMA boxes of 8 channels each),
// B is [k-chunk 2][out-channel 16][8 in-channels] per tap.
#pragma once
#include "hpccg_internal.cuh"
#include "unet_tc.cuh"

namespace hpccg {

constexpr int kConvThreads = 192;
constexpr int kConvStages = 24;
constexpr int kTapBytes = 2 * 128 * 16;  // one k-step of A: 2 boxes x 128 voxels x 16 bytes
constexpr int kWTapBytes = 16 * 16 * 2;  // one tap of B: 16 x 16 BF16
// mbarriers after the stages: full[S], empty[S], acc_full[2], acc_empty[2],
// drain[1], then the 4-byte TMEM address slot (rounded up to 16 bytes).
constexpr int kConvBarBytes = (2 * kConvStages + 5) * 8 + 16;
// Dynamic shared memory of a conv CTA with `nin` input groups.
__host__ __device__ constexpr int conv_smem_bytes(int nin) { return nin * 27 * kWTapBytes + kConvStages * kTapBytes + kConvBarBytes; }

// Row-tile variant for bricks that are one 128-voxel x-row (nx a multiple of
// 128): one TMA box per 8-channel half brings the 3x3 neighbouring rows of
// 130 voxels (the brick plus its x halo) and all 27 taps read that halo tile
// through shifted descriptors: 2 TMA loads per tile and input instead of 54.
constexpr int kRowVox = 130;
constexpr int kRowPlaneBytes = ((9 * kRowVox * 16 + 127) / 128) * 128;  // one 8-channel plane, 128-B aligned
constexpr int kRowStages = 2;
__host__ __device__ constexpr int row_stage_bytes(int nin) { return nin * 2 * kRowPlaneBytes; }
constexpr int kRowBarBytes = (2 * kRowStages + 5) * 8 + 16;
__host__ __device__ constexpr int conv_row_smem_bytes(int nin) {
  return nin * 27 * kWTapBytes + kRowStages * row_stage_bytes(nin) + kRowBarBytes;
}

enum ConvEpi : int {
  kEpiBiasRelu = 0,   // out_bf16 = relu(acc + bias)
  kEpiBias = 1,       // out_bf16 = acc + bias
  kEpiProject = 2,    // out_f32 = proj . relu(acc + bias) + proj_bias
  kEpiRawF32 = 3,     // out_f32 = acc (16 channels)
};

struct ConvGeom {
  int nx, ny, nz, nb;  // volume and batch
  int bx, by, bz;      // brick of 128 voxels
  int tx, ty, tz;      // bricks per dimension
  int ntiles;
};

struct ConvArgs {
  ConvGeom g;
  const __nv_bfloat16 *wpack;  // [nin][27][2][16][8] BF16
  const float *bias;           // [16] (nullable for kEpiRawF32)
  const float *proj;           // [17] for kEpiProject: 16 weights + bias
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
  if (bx * by * bz != 128 || nx % bx || ny % by || nz % bz) return false;
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

int make_act_tmap(CUtensorMap *map, const void *base, const ConvGeom &g, bool row_tile = false);
int launch_conv3_tc(int nin, int epi, const CUtensorMap *maps, const ConvArgs &a, int num_sms, cudaStream_t s);
int launch_conv3_tc_row(int nin, int epi, const CUtensorMap *maps, const ConvArgs &a, int num_sms, cudaStream_t s);
// The row-tile kernel applies when each brick is one full 128-voxel x-row.
inline bool conv_row_ok(const ConvGeom &g) { return g.bx == 128 && g.by == 1 && g.bz == 1; }

}  // namespace hpccg
