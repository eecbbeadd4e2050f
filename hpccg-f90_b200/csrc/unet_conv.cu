// unet_conv.cu -- tcgen05 3x3x3 convolution kernels (layout and roles in
// unet_conv.cuh).  Operand tiles arrive by 1D bulk copies of row-planar spans;
// grid faces are zero-filled with ordinary stores, fenced into the async proxy
// before the tensor cores read them.
#include <stdlib.h>

#include <algorithm>

#include "unet_conv.cuh"

namespace hpccg {

using namespace tc;

struct TileOrigin {
  int b, x0, y0, z0;
};

__device__ __forceinline__ TileOrigin tile_origin(const ConvGeom &g, int t) {
  TileOrigin o;
  int r = t;
  o.x0 = (r % g.tx) * g.bx;
  r /= g.tx;
  o.y0 = (r % g.ty) * g.by;
  r /= g.ty;
  o.z0 = (r % g.tz) * g.bz;
  o.b = r / g.tz;
  return o;
}

// One lane's share of a fetch: the span of `len` units of half h of grid row
// (b, z, y) starting at voxel xs goes to dst.  Units outside the grid are
// zeroed here (generic stores); the in-grid part is described for a later
// bulk copy.
struct Span {
  const __nv_bfloat16 *src;
  uint8_t *dst;
  uint32_t bytes;
  bool zeroed;  // this lane wrote zero fill with ordinary stores
};

__device__ __forceinline__ Span plan_span(const ConvGeom &g, const __nv_bfloat16 *base, int b, int z, int y, int h,
                                          int xs, int len, uint8_t *dst) {
  Span sp{nullptr, nullptr, 0, false};
  const uint4 zero = make_uint4(0, 0, 0, 0);
  if (z < 0 || z >= g.nz || y < 0 || y >= g.ny) {
    for (int u = 0; u < len; ++u) reinterpret_cast<uint4 *>(dst)[u] = zero;
    sp.zeroed = true;
    return sp;
  }
  const int lo = max(xs, 0), hi = min(xs + len, g.nx);
  for (int u = 0; u < lo - xs; ++u) reinterpret_cast<uint4 *>(dst)[u] = zero;
  for (int u = hi - xs; u < len; ++u) reinterpret_cast<uint4 *>(dst)[u] = zero;
  sp.zeroed = lo > xs || hi < xs + len;
  if (hi <= lo) return sp;
  const int64_t row = ((int64_t)b * g.nz + z) * g.ny + y;
  sp.src = base + act_unit(row, h, lo, g.nx) * 8;
  sp.dst = dst + (lo - xs) * 16;
  sp.bytes = (uint32_t)(hi - lo) * 16;
  return sp;
}

// Posts the stage: lanes that zero-filled fence their stores into the async
// proxy, lane 0 arms the barrier with the warp's total bulk bytes, then every
// lane issues its copies.
__device__ __forceinline__ void post_spans(const Span *sp, int nsp, uint64_t *bar, int lane) {
  uint32_t bytes = 0;
  bool zeroed = false;
  for (int i = 0; i < nsp; ++i) {
    bytes += sp[i].bytes;
    zeroed |= sp[i].zeroed;
  }
  if (zeroed) fence_proxy_async_smem();  // only lanes that stored zeros
  const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
  __syncwarp();
  if (lane == 0) mbar_expect_tx(bar, total);
  __syncwarp();
  for (int i = 0; i < nsp; ++i)
    if (sp[i].bytes) bulk_g2s(sp[i].dst, sp[i].src, sp[i].bytes, bar);
}

// Lane 0 waits, the result is shared with the warp.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, int *err, int where, int lane) {
  bool ok = true;
  if (lane == 0) ok = mbar_wait(bar, parity, err, where);
  ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
  __syncwarp();
  return ok;
}

// Epilogue of one voxel: row m of tile t holds its 16 accumulated channels in v.
template <int EPI>
__device__ __forceinline__ void conv_store(const ConvArgs &a, int t, int m, const float *v, const float *bias,
                                           const float *proj) {
  const ConvGeom &g = a.g;
  const TileOrigin o = tile_origin(g, t);
  const int x = o.x0 + m % g.bx, y = o.y0 + (m / g.bx) % g.by, z = o.z0 + m / (g.bx * g.by);
  const int64_t row = ((int64_t)o.b * g.nz + z) * g.ny + y;
  if (EPI == kEpiRawF32) {
    float *out = static_cast<float *>(a.out);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float4 *o4 = reinterpret_cast<float4 *>(out + act_unit(row, h, x, g.nx) * 8);
      o4[0] = make_float4(v[8 * h], v[8 * h + 1], v[8 * h + 2], v[8 * h + 3]);
      o4[1] = make_float4(v[8 * h + 4], v[8 * h + 5], v[8 * h + 6], v[8 * h + 7]);
    }
  } else if (EPI == kEpiProject) {
    float acc = proj[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc = fmaf(proj[c], fmaxf(v[c] + bias[c], 0.f), acc);
    static_cast<float *>(a.out)[row * g.nx + x] = acc;
  } else {
    __nv_bfloat16 *out = static_cast<__nv_bfloat16 *>(a.out);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint32_t w[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float lo = v[8 * h + 2 * c] + bias[8 * h + 2 * c], hi = v[8 * h + 2 * c + 1] + bias[8 * h + 2 * c + 1];
        if (EPI == kEpiBiasRelu) {
          lo = fmaxf(lo, 0.f);
          hi = fmaxf(hi, 0.f);
        }
        const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
        w[c] = *reinterpret_cast<const uint32_t *>(&p);
      }
      *reinterpret_cast<uint4 *>(out + act_unit(row, h, x, g.nx) * 8) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Shared set-up of both kernels: weights to smem, barriers, TMEM (32 columns).
// bars: full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], drain.
template <int NIN, int STAGES>
__device__ __forceinline__ uint32_t conv_setup(const ConvArgs &a, uint8_t *sW, uint64_t *bars, uint32_t *slot,
                                               int warp) {
  constexpr int kWBytes = NIN * 27 * kWTapBytes;
  for (int i = threadIdx.x; i < kWBytes / 16; i += kConvThreads)
    reinterpret_cast<uint4 *>(sW)[i] = reinterpret_cast<const uint4 *>(a.wpack)[i];
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2 * STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_init(&bars[2 * STAGES + 0], 1);
    mbar_init(&bars[2 * STAGES + 1], 1);
    mbar_init(&bars[2 * STAGES + 2], 4);
    mbar_init(&bars[2 * STAGES + 3], 4);
    mbar_init(&bars[2 * STAGES + 4], 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(slot, 32);
    tmem_relinquish();
  }
  fence_proxy_async_smem();  // weights -> tensor-core proxy
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return *slot;
}

// Set-up of the row kernel: weights, the barriers of each of the P pipelines
// (pipeline p starts at rings + p*pipe_bytes; its 2R+5 barriers follow its ring
// of ring_bytes), and
// 32*P TMEM columns allocated by warp 1; the TMEM base lands in *slot.
template <int NIN, int R, int P>
__device__ __forceinline__ uint32_t conv_setup_row(const ConvArgs &a, uint8_t *sW, uint8_t *rings, int ring_bytes,
                                                   int pipe_bytes, uint32_t *slot, int warp) {
  constexpr int kWBytes = NIN * 27 * kWTapBytes;
  for (int i = threadIdx.x; i < kWBytes / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(sW)[i] = reinterpret_cast<const uint4 *>(a.wpack)[i];
  if (threadIdx.x == 0) {
    for (int p = 0; p < P; ++p) {
      uint64_t *bars = reinterpret_cast<uint64_t *>(rings + p * pipe_bytes + ring_bytes);
      for (int s = 0; s < 2 * R; ++s) mbar_init(&bars[s], 1);
      mbar_init(&bars[2 * R + 0], 1);
      mbar_init(&bars[2 * R + 1], 1);
      mbar_init(&bars[2 * R + 2], 4);
      mbar_init(&bars[2 * R + 3], 4);
      mbar_init(&bars[2 * R + 4], 1);
    }
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(slot, 32 * P);
    tmem_relinquish();
  }
  fence_proxy_async_smem();  // weights -> tensor-core proxy
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return *slot;
}

// Epilogue role (warps 2-5): drain each tile's accumulator and store it.
template <int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs &a, uint64_t *acc_full, uint64_t *acc_empty,
                                              uint32_t tmem, int warp, int lane, int where) {
  const int q = warp & 3;
  uint32_t tcount = 0;
  float bias[16], proj[17];
#pragma unroll
  for (int c = 0; c < 16; ++c) bias[c] = (EPI == kEpiRawF32 || !a.bias) ? 0.f : a.bias[c];
  if (EPI == kEpiProject)
#pragma unroll
    for (int c = 0; c < 17; ++c) proj[c] = a.proj[c];
  for (int t = blockIdx.x; t < a.g.ntiles; t += gridDim.x, ++tcount) {
    const int buf = tcount & 1;
    if (!mbar_wait(&acc_full[buf], (tcount >> 1) & 1, a.err, where)) break;
    tc_fence_after();
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 16), v);
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(&acc_empty[buf]);
    conv_store<EPI>(a, t, q * 32 + lane, v, bias, proj);
  }
}

// ---- brick tiles: one fetch per (tap, input) ---------------------------------------------
template <int NIN, int EPI>
__global__ void __launch_bounds__(kConvThreads, 1) k_conv3_brick(ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int kWBytes = NIN * 27 * kWTapBytes;
  constexpr int S = kBrickStages;
  uint8_t *sW = smem;
  uint8_t *sA = smem + kWBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(sA + S * kBrickStageBytes);
  uint64_t *empty = full + S;
  uint64_t *acc_full = empty + S;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain = acc_empty + 2;
  uint32_t *slot = reinterpret_cast<uint32_t *>(drain + 1);
  static_assert((2 * S + 5) * 8 + 4 <= bar_bytes(S), "barrier area");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t tmem = conv_setup<NIN, S>(a, sW, full, slot, warp);
  const ConvGeom &g = a.g;
  constexpr int ksteps = 27 * NIN;

  if (warp == 0) {
    // fetch: 2 halves x by*bz rows per k-step, one span per lane (at most 32)
    const int nrows = g.by * g.bz;
    uint32_t it = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < g.ntiles && ok; t += gridDim.x) {
      const TileOrigin o = tile_origin(g, t);
      for (int ks = 0; ks < ksteps; ++ks, ++it) {
        const int s = it % S;
        const uint32_t n = it / S;
        if (n > 0 && !(ok = warp_wait(&empty[s], (n - 1) & 1, a.err, 1, lane))) break;
        const int tap = ks / NIN, in = ks % NIN;
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        const __nv_bfloat16 *base = (NIN > 1 && in) ? a.in1 : a.in0;
        uint8_t *stage = sA + s * kBrickStageBytes;
        Span sp[1];
        int nsp = 0;
        if (lane < 2 * nrows) {
          const int h = lane / nrows, rr = lane % nrows;
          const int my = rr % g.by, mz = rr / g.by;
          sp[0] = plan_span(g, base, o.b, o.z0 + mz + dz, o.y0 + my + dy, h, o.x0 + dx, g.bx,
                            stage + h * (kBrickStageBytes / 2) + rr * g.bx * 16);
          nsp = 1;
        }
        post_spans(sp, nsp, &full[s], lane);
      }
    }
    if (lane == 0) {  // every issued copy has landed before the CTA may exit
      const uint32_t first = it > (uint32_t)S ? it - S : 0;
      for (uint32_t j = first; j < it; ++j) mbar_wait(&full[j % S], (j / S) & 1, a.err, 5);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16(128, 16);
      const uint64_t ad0 = smem_desc(sA, kBrickStageBytes / 2, 128), wd = smem_desc(sW, 256, 128);
      uint32_t it = 0, tcount = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < g.ntiles && ok; t += gridDim.x, ++tcount) {
        const int buf = tcount & 1;
        const uint32_t use = tcount >> 1;
        if (use > 0 && !(ok = mbar_wait(&acc_empty[buf], (use - 1) & 1, a.err, 2))) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(buf * 16);
        for (int ks = 0; ks < ksteps; ++ks, ++it) {
          const int s = it % S;
          if (!(ok = mbar_wait(&full[s], (it / S) & 1, a.err, 3))) break;
          tc_fence_after();
          const uint64_t ad = ad0 + (uint64_t)((s * kBrickStageBytes) >> 4);
          const uint64_t bd = wd + (uint64_t)((ks % NIN * 27 + ks / NIN) * (kWTapBytes >> 4));
          mma_bf16(d, ad, bd, idesc, ks > 0 ? 1u : 0u);
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(&acc_full[buf]);
      }
      mma_commit(drain);
      mbar_wait(drain, 0, a.err, 6);
    }
  } else {
    conv_epilogue<EPI>(a, acc_full, acc_empty, tmem, warp, lane, 4);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 32);
  }
}

// ---- row tiles: rolling window of slabs along y -------------------------------------------
struct RowUnits {
  int nxb, nchunks, nunits;
};
template <int RX>
__host__ __device__ __forceinline__ RowUnits row_units(const ConvGeom &g) {
  RowUnits r;
  r.nxb = g.nx / RX;
  r.nchunks = (g.ny + row_chunk(RX) - 1) / row_chunk(RX);
  r.nunits = r.nxb * g.nz * g.nb * r.nchunks;
  return r;
}
struct RowUnit {
  int b, z, x0, ya, yb;
};
template <int RX>
__device__ __forceinline__ RowUnit row_unit(const ConvGeom &g, const RowUnits &ru, int u) {
  RowUnit w;
  const int c = u % ru.nchunks;
  int r = u / ru.nchunks;
  w.x0 = (r % ru.nxb) * RX;
  r /= ru.nxb;
  w.z = r % g.nz;
  w.b = r / g.nz;
  w.ya = c * row_chunk(RX);
  w.yb = min(g.ny, w.ya + row_chunk(RX));
  return w;
}
// Tile index (as tile_origin decodes it, g.bx = RX) of row y of a unit.
template <int RX>
__device__ __forceinline__ int row_tile_index(const ConvGeom &g, const RowUnit &w, int y) {
  return ((w.b * g.nz + w.z) * g.ny + y) * g.tx + w.x0 / RX;
}

// RX = 128: one TMEM lane per voxel.  RX = 64 (MMA M = 64): voxel row m of the
// tile sits in TMEM lane (m / 16) * 32 + m % 16, i.e. lanes 0-15 of each
// warp's quarter (checked on the GPU by dumping an M = 64 accumulator).
template <int NIN, int EPI, int RX>
__global__ void __launch_bounds__(kConvThreads * row_pipes(NIN, RX), 1) k_conv3_row(ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int P = row_pipes(NIN, RX);
  constexpr int kWBytes = NIN * 27 * kWTapBytes;
  constexpr int kSlab = slab_bytes(NIN, RX);
  constexpr int R = row_slots(NIN, RX, P);
  constexpr int kRowVox = row_vox(RX), kSlabPlaneBytes = slab_plane_bytes(RX);
  static_assert(RX == 128 || RX == 64, "MMA M is 128 or 64");
  static_assert((2 * R + 5) * 8 + 4 <= bar_bytes(R), "barrier area");
  static_assert(R >= 4, "the window needs the three slabs of a tile plus one in flight");
  constexpr int kPipeBytes = row_pipe_bytes(NIN, RX);
  static_assert(R * kSlab + bar_bytes(R) <= kPipeBytes && kPipeBytes % 128 == 0, "shared memory plan");
  // pipeline `pipe` = warps 6*pipe .. 6*pipe+5 in the roles producer, MMA, 4 x epilogue;
  // it owns units blockIdx.x + (k*P + pipe)*gridDim.x, its slab ring, its barriers
  // and TMEM columns 32*pipe .. +31
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pipe = warp / 6, role = warp % 6;
  uint8_t *sW = smem;
  uint8_t *sA = smem + kWBytes + pipe * kPipeBytes;
  uint64_t *full = reinterpret_cast<uint64_t *>(sA + R * kSlab);
  uint64_t *empty = full + R;
  uint64_t *acc_full = empty + R;
  uint64_t *acc_empty = acc_full + 2;
  uint64_t *drain = acc_empty + 2;
  uint32_t *slot = reinterpret_cast<uint32_t *>(smem + kWBytes + R * kSlab + 2 * R * 8 + 5 * 8);  // pipeline 0's
  const uint32_t tmem = conv_setup_row<NIN, R, P>(a, sW, smem + kWBytes, R * kSlab, kPipeBytes, slot, warp) + 32 * pipe;
  const ConvGeom &g = a.g;
  const RowUnits ru = row_units<RX>(g);
  const int u0 = blockIdx.x + pipe * gridDim.x, ustep = P * gridDim.x;

  if (role == 0) {
    // fetch slabs ya-1 .. yb of every unit: NIN x 2 halves x 3 z-rows spans
    uint32_t sc = 0;
    bool ok = true;
    for (int u = u0; u < ru.nunits && ok; u += ustep) {
      const RowUnit w = row_unit<RX>(g, ru, u);
      for (int ys = w.ya - 1; ys <= w.yb; ++ys, ++sc) {
        const int s = sc % R;
        const uint32_t n = sc / R;
        if (n > 0 && !(ok = warp_wait(&empty[s], (n - 1) & 1, a.err, 11, lane))) break;
        uint8_t *base = sA + s * kSlab;
        Span sp[1];
        int nsp = 0;
        if (lane < 6 * NIN) {
          const int r = lane % 3, h = (lane / 3) & 1, in = lane / 6;
          sp[0] = plan_span(g, in ? a.in1 : a.in0, w.b, w.z + r - 1, ys, h, w.x0 - 1, kRowVox,
                            base + (in * 2 + h) * kSlabPlaneBytes + r * kRowVox * 16);
          nsp = 1;
        }
        post_spans(sp, nsp, &full[s], lane);
      }
    }
    if (lane == 0) {
      const uint32_t first = sc > (uint32_t)R ? sc - R : 0;
      for (uint32_t j = first; j < sc; ++j) mbar_wait(&full[j % R], (j / R) & 1, a.err, 15);
    }
  } else if (role == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16(RX, 16);
      const uint64_t wd = smem_desc(sW, 256, 128);
      uint32_t sc0 = 0, tcount = 0;
      bool ok = true;
      for (int u = u0; u < ru.nunits && ok; u += ustep) {
        const RowUnit w = row_unit<RX>(g, ru, u);
        const int ntile = w.yb - w.ya;
        uint32_t ready = sc0;  // slabs [sc0, ready) have been waited for
        for (int i = 0; i < ntile; ++i, ++tcount) {
          const int buf = tcount & 1;
          const uint32_t use = tcount >> 1;
          if (use > 0 && !(ok = mbar_wait(&acc_empty[buf], (use - 1) & 1, a.err, 12))) break;
          for (; ready < sc0 + i + 3; ++ready)
            if (!(ok = mbar_wait(&full[ready % R], (ready / R) & 1, a.err, 13))) break;
          if (!ok) break;
          tc_fence_after();
          const uint32_t d = tmem + (uint32_t)(buf * 16);
          // descriptors of the three slabs (y-1, y, y+1); a tap adds a constant
          // offset (address field in 16-byte units, no carry: smem < 256 KB)
          uint64_t sd[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) sd[j] = smem_desc(sA + ((sc0 + i + j) % R) * kSlab, kSlabPlaneBytes, 128);
          // taps in dy-major order: the nine of dy = -1 first, so slab y-1 (this
          // tile is its last user) is released as soon as they complete and the
          // producer refills its slot while the other 18 run
#pragma unroll
          for (int ks = 0; ks < 27 * NIN; ++ks) {
            const int t = ks / NIN, in = ks % NIN;
            const int dyp = t / 9, dzp = (t / 3) % 3, dxp = t % 3;  // offsets + 1
            const int tap = dzp * 9 + dyp * 3 + dxp;
            const uint64_t ad = sd[dyp] + (uint64_t)((in * 2 * kSlabPlaneBytes + (dzp * kRowVox + dxp) * 16) >> 4);
            const uint64_t bd = wd + (uint64_t)(((in * 27 + tap) * kWTapBytes) >> 4);
            mma_bf16(d, ad, bd, idesc, ks > 0 ? 1u : 0u);
            if (ks == 9 * NIN - 1) mma_commit(&empty[(sc0 + i) % R]);  // slab y-1 is done for the unit
          }
          mma_commit(&acc_full[buf]);
        }
        if (!ok) break;
        mma_commit(&empty[(sc0 + ntile) % R]);  // the unit's last two slabs
        mma_commit(&empty[(sc0 + ntile + 1) % R]);
        sc0 += ntile + 2;
      }
      mma_commit(drain);
      mbar_wait(drain, 0, a.err, 16);
    }
  } else {
    // epilogue: tiles in unit order
    const int q = warp & 3;
    uint32_t tcount = 0;
    float bias[16], proj[17];
#pragma unroll
    for (int c = 0; c < 16; ++c) bias[c] = (EPI == kEpiRawF32 || !a.bias) ? 0.f : a.bias[c];
    if (EPI == kEpiProject)
#pragma unroll
      for (int c = 0; c < 17; ++c) proj[c] = a.proj[c];
    bool ok = true;
    for (int u = u0; u < ru.nunits && ok; u += ustep) {
      const RowUnit w = row_unit<RX>(g, ru, u);
      for (int y = w.ya; y < w.yb; ++y, ++tcount) {
        const int buf = tcount & 1;
        if (!(ok = mbar_wait(&acc_full[buf], (tcount >> 1) & 1, a.err, 14))) break;
        tc_fence_after();
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 16), v);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[buf]);
        if (RX == 128)
          conv_store<EPI>(a, row_tile_index<RX>(g, w, y), q * 32 + lane, v, bias, proj);
        else if (lane < 16)
          conv_store<EPI>(a, row_tile_index<RX>(g, w, y), q * 16 + lane, v, bias, proj);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem - 32 * pipe, 32 * P);
  }
}

// ---- the 1-channel input layer on tcgen05 (nx a multiple of 128) -------------------------
// An im2col GEMM per tile of 128 voxels of one x row: A[m][k] = in(x0+m+dx, y+dy, z+dz)
// in BF16 for tap k = (dz+1)*9 + (dy+1)*3 + (dx+1) (k = 27..31 zero), B[c][k] = W[k][c];
// two MMAs (M = 128, N = 16, K = 16) into a 16-column FP32 accumulator.  A CTA walks a
// contiguous range of tiles.  The tile's nine input lines (dz, dy), x0-1 .. x0+128 with
// zeros outside the grid, are staged once in shared memory: each thread loads one element
// of every line a tile ahead into registers and stores them while the current tile is
// built.  Thread m then reads its voxel's 27 taps from the staged lines into its A row;
// thread 0 issues the tile's MMAs; every warp drains its TMEM lane quarter of the PREVIOUS
// tile (bias, ReLU, BF16 stores), so a tile's MMAs run while the next tile is built.  The
// staged lines, A and the accumulator are double-buffered: one barrier per tile.
constexpr int kIn1Threads = 128;
constexpr int kIn1ABytes = 4 * 128 * 16;  // [4 K chunks of 8 taps][128 rows][8 BF16]
constexpr int kIn1BBytes = 4 * 16 * 16;   // [4 K chunks][16 output channels][8 BF16]
constexpr int kIn1Line = 132;             // a staged line: x0-1+i at [i], i < 130

// tile coordinates in tile order: row = (b*nz + z)*ny + y, x block xb (tile = row*tx + xb)
struct In1Tile {
  int row, xb, y, z;
  __device__ __forceinline__ void at(int t, int tx, int ny, int nz) {
    row = t / tx;
    xb = t - row * tx;
    const int yz = row / ny;
    y = row - yz * ny;
    z = yz % nz;
  }
  __device__ __forceinline__ void next(int tx, int ny, int nz) {
    if (++xb == tx) {
      xb = 0;
      ++row;
      if (++y == ny) {
        y = 0;
        if (++z == nz) z = 0;
      }
    }
  }
};

__global__ void __launch_bounds__(kIn1Threads) k_conv3_in1_tc(const float *in, const float *W, const float *bias,
                                                              __nv_bfloat16 *out, int nx, int ny, int nz, int nb,
                                                              int relu, int *err) {
  __shared__ __align__(1024) uint8_t sA[2][kIn1ABytes];
  __shared__ __align__(128) uint8_t sB[kIn1BBytes];
  __shared__ __align__(16) float sL[2][9 * kIn1Line];
  __shared__ __align__(16) float sBias[16];
  __shared__ uint64_t done[2], fin;
  __shared__ uint32_t slot;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < 32 * 16; e += kIn1Threads) {  // B element (k, c): chunk k/8, row c, position k%8
    const int k = e / 16, c = e % 16;
    reinterpret_cast<__nv_bfloat16 *>(sB)[((k >> 3) * 16 + c) * 8 + (k & 7)] =
        __float2bfloat16(k < 27 ? W[k * 16 + c] : 0.f);
  }
  if (tid < 16) sBias[tid] = bias[tid];
  // tile t = ((b*nz + z)*ny + y)*tx + x-block; 32-bit indices (a grid has fewer than 2^31 tiles)
  const int tx = nx / 128;
  const int ntiles = tx * ny * nz * nb;
  const int t_lo = (int)((int64_t)blockIdx.x * ntiles / gridDim.x);
  const int t_hi = (int)((int64_t)(blockIdx.x + 1) * ntiles / gridDim.x);
  // this thread's element of each staged line (x0 + tid), and for threads 0..8 / 32..40
  // the left / right halo element (x0 - 1 / x0 + 128) of line hl
  const int hl = tid < 9 ? tid : (tid >= 32 && tid < 41 ? tid - 32 : -1);
  const int hx = tid < 32 ? -1 : 128;
  float ld[9], lh = 0.f;
  In1Tile L, D;  // the next tile to load, the next tile to drain
  L.at(t_lo, tx, ny, nz);
  D = L;
  auto load = [&](bool live) {
    const int x0 = L.xb * 128;
#pragma unroll
    for (int l = 0; l < 9; ++l) {
      const int dz = l / 3 - 1, dy = l % 3 - 1;
      const bool ok = live && (unsigned)(L.z + dz) < (unsigned)nz && (unsigned)(L.y + dy) < (unsigned)ny;
      ld[l] = ok ? __ldg(in + (int64_t)(L.row + dz * ny + dy) * nx + x0 + tid) : 0.f;
    }
    if (hl >= 0) {
      const int dz = hl / 3 - 1, dy = hl % 3 - 1, xh = x0 + hx;
      const bool ok = live && (unsigned)(L.z + dz) < (unsigned)nz && (unsigned)(L.y + dy) < (unsigned)ny &&
                      (unsigned)xh < (unsigned)nx;
      lh = ok ? __ldg(in + (int64_t)(L.row + dz * ny + dy) * nx + xh) : 0.f;
    }
    L.next(tx, ny, nz);
  };
  auto stage = [&](int sb) {
    float *s = sL[sb];
#pragma unroll
    for (int l = 0; l < 9; ++l) s[l * kIn1Line + tid + 1] = ld[l];
    if (hl >= 0) s[hl * kIn1Line + hx + 1] = lh;
  };
  load(t_lo < t_hi);
  stage(0);
  load(t_lo + 1 < t_hi);
  if (tid == 0) {
    mbar_init(&done[0], 1);
    mbar_init(&done[1], 1);
    mbar_init(&fin, 1);
    fence_mbar_init();
    s_fail = 0;
  }
  if (warp == 0) {
    tmem_alloc(&slot, 32);
    tmem_relinquish();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();  // B, the bias, the first tile's lines, the barriers and the TMEM slot
  tc_fence_after();
  const uint32_t tmem = slot;
  constexpr uint32_t idesc = idesc_bf16(128, 16);
  const uint64_t bd = smem_desc(sB, 256, 128);
  // the epilogue of tile D (buffer buf, its use u of that buffer): bias, ReLU, BF16 stores
  auto drain = [&](int buf, uint32_t use) {
    if (!mbar_wait(&done[buf], use & 1u, err, 31)) s_fail = 1;
    tc_fence_after();
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * 16), v);
    tc_fence_before();
    const int x = D.xb * 128 + tid;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float4 b0 = *reinterpret_cast<const float4 *>(sBias + 8 * h);
      const float4 b1 = *reinterpret_cast<const float4 *>(sBias + 8 * h + 4);
      const float bc[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
      uint32_t w[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float lo = v[8 * h + 2 * c] + bc[2 * c], hi = v[8 * h + 2 * c + 1] + bc[2 * c + 1];
        if (relu) {
          lo = fmaxf(lo, 0.f);
          hi = fmaxf(hi, 0.f);
        }
        const __nv_bfloat162 pr = __floats2bfloat162_rn(lo, hi);
        w[c] = *reinterpret_cast<const uint32_t *>(&pr);
      }
      *reinterpret_cast<uint4 *>(out + act_unit(D.row, h, x, nx) * 8) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    D.next(tx, ny, nz);
  };
  int it = 0;
  for (int t = t_lo; t < t_hi; ++t, ++it) {
    const int buf = it & 1;
    // this thread's voxel: 27 taps from the staged lines
    const float *s = sL[buf] + tid;
    float v[32];
#pragma unroll
    for (int l = 0; l < 9; ++l)
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) v[l * 3 + dx] = s[l * kIn1Line + dx];
#pragma unroll
    for (int k = 27; k < 32; ++k) v[k] = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const __nv_bfloat162 pr = __floats2bfloat162_rn(v[8 * c + 2 * j], v[8 * c + 2 * j + 1]);
        w[j] = *reinterpret_cast<const uint32_t *>(&pr);
      }
      *reinterpret_cast<uint4 *>(sA[buf] + c * 2048 + (tid >> 3) * 128 + (tid & 7) * 16) =
          make_uint4(w[0], w[1], w[2], w[3]);
    }
    stage(buf ^ 1);        // tile t+1's lines: that buffer was last read before the previous barrier
    load(t + 2 < t_hi);    // tile t+2's elements, in flight until the next iteration's stage
    fence_proxy_async_smem();  // the A rows -> tensor-core proxy
    tc_fence_before();
    __syncthreads();  // A and the next lines written; the drain of this buffer's last tile is done
    tc_fence_after();
    if (s_fail) break;  // read by every thread after the same barrier
    if (tid == 0) {
      const uint64_t ad = smem_desc(sA[buf], 2048, 128);
      const uint32_t d = tmem + (uint32_t)(buf * 16);
      mma_bf16(d, ad, bd, idesc, 0u);
      mma_bf16(d, ad + (uint64_t)(4096 >> 4), bd + (uint64_t)(512 >> 4), idesc, 1u);
      mma_commit(&done[buf]);
    }
    if (it > 0) drain(buf ^ 1, (uint32_t)((it - 1) >> 1));
  }
  if (it > 0 && !s_fail) drain((it - 1) & 1, (uint32_t)((it - 1) >> 1));
  if (tid == 0) {  // every MMA this thread issued has completed before TMEM is freed
    mma_commit(&fin);
    mbar_wait(&fin, 0, err, 32);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, 32);
  }
}

int launch_conv3_in1_tc(const float *in, const float *W, const float *bias, __nv_bfloat16 *out, int nx, int ny,
                        int nz, int nb, int relu, int *err, int num_sms, cudaStream_t s) {
  if (nx % 128 || ny < 1 || nz < 1 || nb < 1) return HPCCG_ERR_UNSUPPORTED;
  const int64_t ntiles = (int64_t)(nx / 128) * ny * nz * nb;
  if (ntiles >= ((int64_t)1 << 31)) return HPCCG_ERR_TOO_LARGE;
  const int grid = (int)std::min<int64_t>(ntiles, (int64_t)num_sms * 8);
  k_conv3_in1_tc<<<grid, kIn1Threads, 0, s>>>(in, W, bias, out, nx, ny, nz, nb, relu, err);
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

// RX = 0: brick tiles; 128 / 64: row tiles of that many voxels.
template <int NIN, int EPI, int RX>
static int launch_one(const ConvArgs &a, int num_sms, cudaStream_t s) {
  constexpr bool ROW = RX != 0;
  constexpr int smem = ROW ? row_smem_bytes(NIN, RX == 0 ? 128 : RX) : brick_smem_bytes(NIN);
  static_assert(smem <= 227 * 1024, "conv CTA exceeds the shared-memory limit");
  auto kern = ROW ? k_conv3_row<NIN, EPI, RX == 0 ? 128 : RX> : k_conv3_brick<NIN, EPI>;
  static int per_sm = 0;
  if (!per_sm) {
    HPCCG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // resident CTAs per SM by shared memory (each CTA also reserves 1 KB)
    per_sm = std::max(1, (227 * 1024) / (smem + 1024));
  }
  constexpr int pipes = ROW ? row_pipes(NIN, RX == 0 ? 128 : RX) : 1;
  const int work = ROW ? row_units<RX == 0 ? 128 : RX>(a.g).nunits : a.g.ntiles;
  const int grid = std::min((work + pipes - 1) / pipes, num_sms * per_sm);
  kern<<<grid, kConvThreads * pipes, smem, s>>>(a);
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

template <int NIN, int EPI>
static int launch_mode(const ConvArgs &a, int num_sms, cudaStream_t s, int rx) {
  if (rx == 128) return launch_one<NIN, EPI, 128>(a, num_sms, s);
  if (rx == 64) return launch_one<NIN, EPI, 64>(a, num_sms, s);
  return launch_one<NIN, EPI, 0>(a, num_sms, s);
}

int launch_conv3_tc(int nin, int epi, const ConvArgs &a_in, int num_sms, cudaStream_t s, bool force_brick) {
  ConvArgs a = a_in;
  int row = 0;
  if (!force_brick) {
    ConvGeom g64;
    if (conv_row_ok(a.g)) {
      row = 128;
    } else if (conv_row64_geom(a.g, &g64)) {
      a.g = g64;
      row = 64;
    }
  }
  if (nin == 1) {
    switch (epi) {
      case kEpiBiasRelu: return launch_mode<1, kEpiBiasRelu>(a, num_sms, s, row);
      case kEpiBias: return launch_mode<1, kEpiBias>(a, num_sms, s, row);
      case kEpiProject: return launch_mode<1, kEpiProject>(a, num_sms, s, row);
      default: return launch_mode<1, kEpiRawF32>(a, num_sms, s, row);
    }
  }
  switch (epi) {
    case kEpiBiasRelu: return launch_mode<2, kEpiBiasRelu>(a, num_sms, s, row);
    case kEpiBias: return launch_mode<2, kEpiBias>(a, num_sms, s, row);
    case kEpiProject: return launch_mode<2, kEpiProject>(a, num_sms, s, row);
    default: return launch_mode<2, kEpiRawF32>(a, num_sms, s, row);
  }
}

}  // namespace hpccg
