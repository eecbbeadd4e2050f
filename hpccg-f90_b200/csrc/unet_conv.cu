// unet_conv.cu -- the U-Net's 3x3x3 convolution kernels.
//
//  k_conv3_tc<NIN, EPI>: tcgen05/TMA implicit GEMM (see unet_conv.cuh), used
//      for every 16-channel conv on volumes of >= 128 voxels, forward and
//      backward-data (flipped, transposed weights).
//  k_conv3_cc: CUDA-core direct conv (FP32 accumulate) for the 1-channel input
//      layer and volumes smaller than one 128-voxel brick.
#include <cudaTypedefs.h>
#include <stdlib.h>

#include <mutex>

#include "unet_conv.cuh"

namespace hpccg {

using namespace tc;

// Epilogue of one voxel: row m of tile t holds its 16 accumulated channels in v.
template <int EPI>
__device__ __forceinline__ void conv_store(const ConvArgs &a, int t, int m, const float *v, const float *bias,
                                           const float *proj) {
  const ConvGeom &g = a.g;
  int r = t;
  const int x0 = (r % g.tx) * g.bx;
  r /= g.tx;
  const int y0 = (r % g.ty) * g.by;
  r /= g.ty;
  const int z0 = (r % g.tz) * g.bz;
  const int b = r / g.tz;
  const int x = x0 + m % g.bx, y = y0 + (m / g.bx) % g.by, z = z0 + m / (g.bx * g.by);
  const size_t vox = (((size_t)b * g.nz + z) * g.ny + y) * g.nx + x;
  if (EPI == kEpiRawF32) {
    float4 *o = reinterpret_cast<float4 *>(static_cast<float *>(a.out) + vox * 16);
#pragma unroll
    for (int c = 0; c < 4; ++c) o[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
  } else if (EPI == kEpiProject) {
    float acc = proj[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc = fmaf(proj[c], fmaxf(v[c] + bias[c], 0.f), acc);
    static_cast<float *>(a.out)[vox] = acc;
  } else {
    uint32_t w[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float lo = v[2 * c] + bias[2 * c], hi = v[2 * c + 1] + bias[2 * c + 1];
      if (EPI == kEpiBiasRelu) {
        lo = fmaxf(lo, 0.f);
        hi = fmaxf(hi, 0.f);
      }
      const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
      w[c] = *reinterpret_cast<const uint32_t *>(&h);
    }
    uint4 *o = reinterpret_cast<uint4 *>(static_cast<__nv_bfloat16 *>(a.out) + vox * 16);
    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

template <int NIN, int EPI>
__global__ void __launch_bounds__(kConvThreads, 1)
    k_conv3_tc(const __grid_constant__ CUtensorMap map0, const __grid_constant__ CUtensorMap map1, ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int kWBytes = NIN * 27 * kWTapBytes;
  uint8_t *sW = smem;
  uint8_t *sA = smem + kWBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(sA + kConvStages * kTapBytes);
  uint64_t *empty = full + kConvStages;
  uint64_t *acc_full = empty + kConvStages;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain = acc_empty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  static_assert((2 * kConvStages + 5) * 8 + 4 <= kConvBarBytes, "barrier area");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kWBytes / 16; i += kConvThreads)
    reinterpret_cast<uint4 *>(sW)[i] = reinterpret_cast<const uint4 *>(a.wpack)[i];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kConvStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 32);
    tmem_relinquish();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // weights -> tensor-core proxy
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const ConvGeom &g = a.g;
  constexpr int ksteps = 27 * NIN;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    prefetch_tmap(&map0);
    if (NIN > 1) prefetch_tmap(&map1);
    uint32_t it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < g.ntiles && ok; t += gridDim.x) {
      int r = t;
      const int x0 = (r % g.tx) * g.bx;
      r /= g.tx;
      const int y0 = (r % g.ty) * g.by;
      r /= g.ty;
      const int z0 = (r % g.tz) * g.bz;
      const int b = r / g.tz;
      for (int ks = 0; ks < ksteps; ++ks, ++it) {
        const int s = it % kConvStages;
        const uint32_t n = it / kConvStages;
        if (n > 0 && !(ok = mbar_wait(&empty[s], (n - 1) & 1, a.err, 1))) break;
        const int tap = ks / NIN, in = ks % NIN;
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        const CUtensorMap *m = (NIN > 1 && in) ? &map1 : &map0;
        uint8_t *dst = sA + s * kTapBytes;
        mbar_expect_tx(&full[s], kTapBytes);
        tma_load_5d(dst, m, &full[s], 0, x0 + dx, y0 + dy, z0 + dz, b);
        tma_load_5d(dst + kTapBytes / 2, m, &full[s], 8, x0 + dx, y0 + dy, z0 + dz, b);
      }
    }
    // drain: every issued load has landed before the CTA may exit
    const uint32_t first = it > (uint32_t)kConvStages ? it - kConvStages : 0;
    for (uint32_t j = first; j < it; ++j) mbar_wait(&full[j % kConvStages], (j / kConvStages) & 1, a.err, 5);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    constexpr uint32_t idesc = idesc_bf16(128, 16);
    uint32_t it = 0, tcount = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < g.ntiles && ok; t += gridDim.x, ++tcount) {
      const int buf = tcount & 1;
      const uint32_t use = tcount >> 1;
      if (use > 0 && !(ok = mbar_wait(&acc_empty[buf], (use - 1) & 1, a.err, 2))) break;
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(buf * 16);
      for (int ks = 0; ks < ksteps; ++ks, ++it) {
        const int s = it % kConvStages;
        if (!(ok = mbar_wait(&full[s], (it / kConvStages) & 1, a.err, 3))) break;
        tc_fence_after();
        const int tap = ks / NIN, in = ks % NIN;
        const uint64_t ad = smem_desc(sA + s * kTapBytes, kTapBytes / 2, 128);
        const uint64_t bd = smem_desc(sW + (in * 27 + tap) * kWTapBytes, 256, 128);
        mma_bf16(d, ad, bd, idesc, ks > 0 ? 1u : 0u);
        mma_commit(&empty[s]);
      }
      if (!ok) break;
      mma_commit(&acc_full[buf]);
    }
    mma_commit(drain);  // all MMAs of this thread complete before TMEM is freed
    mbar_wait(drain, 0, a.err, 6);
  } else if (warp >= 2) {
    // ---- epilogue: one TMEM lane (= one voxel) per thread ----
    const int q = warp & 3;
    uint32_t tcount = 0;
    float bias[16], proj[17];
#pragma unroll
    for (int c = 0; c < 16; ++c) bias[c] = (EPI == kEpiRawF32 || !a.bias) ? 0.f : a.bias[c];
    if (EPI == kEpiProject)
#pragma unroll
      for (int c = 0; c < 17; ++c) proj[c] = a.proj[c];
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, ++tcount) {
      const int buf = tcount & 1;
      if (!mbar_wait(&acc_full[buf], (tcount >> 1) & 1, a.err, 4)) break;
      tc_fence_after();
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 16), v);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
      conv_store<EPI>(a, t, q * 32 + lane, v, bias, proj);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 32);
  }
}


// Row-tile conv (bx = 128, by = bz = 1): see kRowVox in unet_conv.cuh.
template <int NIN, int EPI>
__global__ void __launch_bounds__(kConvThreads, 1)
    k_conv3_tc_row(const __grid_constant__ CUtensorMap map0, const __grid_constant__ CUtensorMap map1, ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int kWBytes = NIN * 27 * kWTapBytes;
  constexpr int kStage = row_stage_bytes(NIN);
  uint8_t *sW = smem;
  uint8_t *sA = smem + kWBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(sA + kRowStages * kStage);
  uint64_t *empty = full + kRowStages;
  uint64_t *acc_full = empty + kRowStages;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain = acc_empty + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);
  static_assert((2 * kRowStages + 5) * 8 + 4 <= kRowBarBytes, "barrier area");
  static_assert(kWBytes % 128 == 0 && kStage % 128 == 0, "TMA destinations must be 128-byte aligned");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kWBytes / 16; i += kConvThreads)
    reinterpret_cast<uint4 *>(sW)[i] = reinterpret_cast<const uint4 *>(a.wpack)[i];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kRowStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(drain, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 32);
    tmem_relinquish();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const ConvGeom &g = a.g;
  constexpr uint32_t kTx = NIN * 2 * 9 * kRowVox * 16;  // bytes the TMA boxes write per stage

  if (warp == 0 && lane == 0) {
    prefetch_tmap(&map0);
    if (NIN > 1) prefetch_tmap(&map1);
    uint32_t it = 0;
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, ++it) {
      const int s = it % kRowStages;
      const uint32_t n = it / kRowStages;
      if (n > 0 && !mbar_wait(&empty[s], (n - 1) & 1, a.err, 11)) break;
      int r = t;
      const int x0 = (r % g.tx) * 128;
      r /= g.tx;
      const int y0 = r % g.ny;
      r /= g.ny;
      const int z0 = r % g.nz;
      const int b = r / g.nz;
      uint8_t *dst = sA + s * kStage;
      mbar_expect_tx(&full[s], kTx);
      for (int in = 0; in < NIN; ++in) {
        const CUtensorMap *m = in ? &map1 : &map0;
        tma_load_5d(dst + (in * 2 + 0) * kRowPlaneBytes, m, &full[s], 0, x0 - 1, y0 - 1, z0 - 1, b);
        tma_load_5d(dst + (in * 2 + 1) * kRowPlaneBytes, m, &full[s], 8, x0 - 1, y0 - 1, z0 - 1, b);
      }
    }
    const uint32_t first = it > (uint32_t)kRowStages ? it - kRowStages : 0;
    for (uint32_t j = first; j < it; ++j) mbar_wait(&full[j % kRowStages], (j / kRowStages) & 1, a.err, 15);
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t idesc = idesc_bf16(128, 16);
    uint32_t tcount = 0;
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, ++tcount) {
      const int s = tcount % kRowStages;
      const int buf = tcount & 1;
      const uint32_t use = tcount >> 1;
      if (use > 0 && !mbar_wait(&acc_empty[buf], (use - 1) & 1, a.err, 12)) break;
      if (!mbar_wait(&full[s], (tcount / kRowStages) & 1, a.err, 13)) break;
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(buf * 16);
      const uint8_t *stage = sA + s * kStage;
#pragma unroll 1
      for (int ks = 0; ks < 27 * NIN; ++ks) {
        const int tap = ks / NIN, in = ks % NIN;
        const int row = (tap / 9) * 3 + (tap / 3) % 3;  // (dz+1)*3 + (dy+1)
        const int dxp = tap % 3;                         // dx + 1
        const uint8_t *ap = stage + in * 2 * kRowPlaneBytes + (row * kRowVox + dxp) * 16;
        const uint64_t ad = smem_desc(ap, kRowPlaneBytes, 128);
        const uint64_t bd = smem_desc(sW + (in * 27 + tap) * kWTapBytes, 256, 128);
        mma_bf16(d, ad, bd, idesc, ks > 0 ? 1u : 0u);
      }
      mma_commit(&empty[s]);
      mma_commit(&acc_full[buf]);
    }
    mma_commit(drain);
    mbar_wait(drain, 0, a.err, 16);
  } else if (warp >= 2) {
    const int q = warp & 3;
    uint32_t tcount = 0;
    float bias[16], proj[17];
#pragma unroll
    for (int c = 0; c < 16; ++c) bias[c] = (EPI == kEpiRawF32 || !a.bias) ? 0.f : a.bias[c];
    if (EPI == kEpiProject)
#pragma unroll
      for (int c = 0; c < 17; ++c) proj[c] = a.proj[c];
    for (int t = blockIdx.x; t < g.ntiles; t += gridDim.x, ++tcount) {
      const int buf = tcount & 1;
      if (!mbar_wait(&acc_full[buf], (tcount >> 1) & 1, a.err, 14)) break;
      tc_fence_after();
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 16), v);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[buf]);
      conv_store<EPI>(a, t, q * 32 + lane, v, bias, proj);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 32);
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::mutex g_encode_mu;

static int get_encoder() {
  std::lock_guard<std::mutex> lk(g_encode_mu);
  if (g_encode) return HPCCG_OK;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
    return set_cuda_error(e == cudaSuccess ? cudaErrorNotSupported : e, "cuTensorMapEncodeTiled", __FILE__, __LINE__);
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return HPCCG_OK;
}

// Tensor map over a channels-last BF16 activation [nb][nz][ny][nx][16]; box =
// 8 channels x one 128-voxel brick, zero fill outside the volume.
int make_act_tmap(CUtensorMap *map, const void *base, const ConvGeom &g, bool row_tile) {
  int rc = get_encoder();
  if (rc) return rc;
  const cuuint64_t dims[5] = {16, (cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)g.nb};
  const cuuint64_t strides[4] = {32, (cuuint64_t)g.nx * 32, (cuuint64_t)g.nx * g.ny * 32,
                                 (cuuint64_t)g.nx * g.ny * g.nz * 32};
  // row tiles: 8 channels x (128 + 2) voxels x 3 rows x 3 planes (the halo tile)
  const cuuint32_t box[5] = {8, row_tile ? (cuuint32_t)kRowVox : (cuuint32_t)g.bx, row_tile ? 3u : (cuuint32_t)g.by,
                             row_tile ? 3u : (cuuint32_t)g.bz, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(base), dims, strides,
                              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HPCCG_OK : HPCCG_ERR_INVALID_ARG;
}

template <int NIN, int EPI>
static int launch_one(const CUtensorMap *maps, const ConvArgs &a, int num_sms, cudaStream_t s) {
  constexpr size_t smem = conv_smem_bytes(NIN);
  static_assert(conv_smem_bytes(NIN) <= 227 * 1024, "conv CTA exceeds the shared-memory limit");
  static int per_sm = 0;
  if (!per_sm) {
    HPCCG_CUDA(cudaFuncSetAttribute(k_conv3_tc<NIN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HPCCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3_tc<NIN, EPI>, kConvThreads, smem));
    if (per_sm < 1) per_sm = 1;
  }
  // every resident CTA keeps kConvStages TMA loads in flight
  const int grid = std::min(a.g.ntiles, num_sms * per_sm);
  k_conv3_tc<NIN, EPI><<<grid, kConvThreads, smem, s>>>(maps[0], NIN > 1 ? maps[1] : maps[0], a);
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

template <int NIN, int EPI>
static int launch_row(const CUtensorMap *maps, const ConvArgs &a, int num_sms, cudaStream_t s) {
  constexpr size_t smem = conv_row_smem_bytes(NIN);
  static_assert(conv_row_smem_bytes(NIN) <= 227 * 1024, "row conv CTA exceeds the shared-memory limit");
  static int per_sm = 0;
  if (!per_sm) {
    HPCCG_CUDA(cudaFuncSetAttribute(k_conv3_tc_row<NIN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HPCCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3_tc_row<NIN, EPI>, kConvThreads, smem));
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = std::min(a.g.ntiles, num_sms * per_sm);
  k_conv3_tc_row<NIN, EPI><<<grid, kConvThreads, smem, s>>>(maps[0], NIN > 1 ? maps[1] : maps[0], a);
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

int launch_conv3_tc_row(int nin, int epi, const CUtensorMap *maps, const ConvArgs &a, int num_sms, cudaStream_t s) {
  if (nin == 1) {
    switch (epi) {
      case kEpiBiasRelu: return launch_row<1, kEpiBiasRelu>(maps, a, num_sms, s);
      case kEpiBias: return launch_row<1, kEpiBias>(maps, a, num_sms, s);
      case kEpiProject: return launch_row<1, kEpiProject>(maps, a, num_sms, s);
      default: return launch_row<1, kEpiRawF32>(maps, a, num_sms, s);
    }
  }
  switch (epi) {
    case kEpiBiasRelu: return launch_row<2, kEpiBiasRelu>(maps, a, num_sms, s);
    case kEpiBias: return launch_row<2, kEpiBias>(maps, a, num_sms, s);
    case kEpiProject: return launch_row<2, kEpiProject>(maps, a, num_sms, s);
    default: return launch_row<2, kEpiRawF32>(maps, a, num_sms, s);
  }
}

int launch_conv3_tc(int nin, int epi, const CUtensorMap *maps, const ConvArgs &a, int num_sms, cudaStream_t s) {
  if (nin == 1) {
    switch (epi) {
      case kEpiBiasRelu: return launch_one<1, kEpiBiasRelu>(maps, a, num_sms, s);
      case kEpiBias: return launch_one<1, kEpiBias>(maps, a, num_sms, s);
      case kEpiProject: return launch_one<1, kEpiProject>(maps, a, num_sms, s);
      default: return launch_one<1, kEpiRawF32>(maps, a, num_sms, s);
    }
  }
  switch (epi) {
    case kEpiBiasRelu: return launch_one<2, kEpiBiasRelu>(maps, a, num_sms, s);
    case kEpiBias: return launch_one<2, kEpiBias>(maps, a, num_sms, s);
    case kEpiProject: return launch_one<2, kEpiProject>(maps, a, num_sms, s);
    default: return launch_one<2, kEpiRawF32>(maps, a, num_sms, s);
  }
}

}  // namespace hpccg
