// unet_ops.cu -- CUDA-core kernels of the U-Net: the 1-channel input conv and
// small-volume convs, weight packing for the tcgen05 convs, pooling,
// upsampling, ReLU masks, weight/bias gradients, the output projection, the
// loss and the Adam update.  All are memory-bound or tiny.  16-channel
// tensors use the row-planar layout of unet_conv.cuh (act_unit / act_elem).
#include "unet_ops.cuh"

namespace hpccg {

// ---- weight packing ------------------------------------------------------------------
// Forward B operand of input group `in`: packed[in][tap][kc][co][j] =
// W[tap][in*16 + kc*8 + j][co] (W is FP32 [27][cin][16]).
__global__ void k_pack_fwd(const float *W, int cin, int nin, __nv_bfloat16 *packed) {
  const int total = nin * 27 * 256;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int j = e & 7, co = (e >> 3) & 15, kc = (e >> 7) & 1, tap = (e >> 8) % 27, in = (e >> 8) / 27;
    packed[e] = __float2bfloat16(W[((size_t)tap * cin + in * 16 + kc * 8 + j) * 16 + co]);
  }
}
// Backward-data operand for the gradient w.r.t. input group g: a conv over dY
// (16 channels) with taps flipped and in/out transposed:
// packed[tap][kc][ci][j] = W[26 - tap][g*16 + ci][kc*8 + j].
__global__ void k_pack_bwd(const float *W, int cin, int g, __nv_bfloat16 *packed) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 27 * 256; e += gridDim.x * blockDim.x) {
    const int j = e & 7, ci = (e >> 3) & 15, kc = (e >> 7) & 1, tap = e >> 8;
    packed[e] = __float2bfloat16(W[((size_t)(26 - tap) * cin + g * 16 + ci) * 16 + kc * 8 + j]);
  }
}
// The same flipped/transposed weights in FP32 [27][16][16] for the CUDA-core conv.
__global__ void k_flip_fp32(const float *W, int cin, int g, float *Wf) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 27 * 256; e += gridDim.x * blockDim.x) {
    const int ci = e & 15, co = (e >> 4) & 15, tap = e >> 8;  // Wf[tap][co as input][ci as output]
    Wf[e] = W[((size_t)(26 - tap) * cin + g * 16 + ci) * 16 + co];
  }
}

// ---- direct conv on CUDA cores --------------------------------------------------------
// out[v][co] = sum_tap sum_ci in[v + off(tap)][ci] * W[tap][ci][co] (+ bias, ReLU).
// Inputs: in0/in1 row-planar BF16 16-channel tensors (in1 nullable), or in_f32
// one-channel FP32 (cin = 1).  One thread per output voxel.
__global__ void k_conv3_cc(CcConvArgs a) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int64_t nvox = (int64_t)nx * ny * nz * a.nb;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)((v / ((int64_t)nx * ny)) % nz);
    const int64_t b = v / ((int64_t)nx * ny * nz);
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c] = 0.f;
    for (int tap = 0; tap < 27; ++tap) {
      const int xx = x + tap % 3 - 1, yy = y + (tap / 3) % 3 - 1, zz = z + tap / 9 - 1;
      if (xx < 0 || xx >= nx || yy < 0 || yy >= ny || zz < 0 || zz >= nz) continue;
      const int64_t row = (b * nz + zz) * ny + yy;
      if (a.in_f32) {
        const float s = a.in_f32[row * nx + xx];
        const float *w = a.W + (size_t)tap * 16;
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = fmaf(s, w[c], acc[c]);
        continue;
      }
      for (int g = 0; g < a.nin; ++g) {
        const __nv_bfloat16 *src = g ? a.in1 : a.in0;
        for (int ci = 0; ci < 16; ++ci) {
          const float s = __bfloat162float(src[act_elem(row, xx, ci, nx)]);
          const float *w = a.W + ((size_t)tap * a.cin + g * 16 + ci) * 16;
#pragma unroll
          for (int c = 0; c < 16; ++c) acc[c] = fmaf(s, w[c], acc[c]);
        }
      }
    }
    const int64_t orow = (b * nz + z) * ny + y;
    if (a.epi == kEpiRawF32) {
      float *o = static_cast<float *>(a.out);
#pragma unroll
      for (int c = 0; c < 16; ++c) o[act_elem(orow, x, c, nx)] = acc[c];
    } else if (a.epi == kEpiProject) {
      float r = a.proj[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) r = fmaf(a.proj[c], fmaxf(acc[c] + a.bias[c], 0.f), r);
      static_cast<float *>(a.out)[v] = r;
    } else {
      __nv_bfloat16 *o = static_cast<__nv_bfloat16 *>(a.out);
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        float t = acc[c] + (a.bias ? a.bias[c] : 0.f);
        if (a.epi == kEpiBiasRelu) t = fmaxf(t, 0.f);
        o[act_elem(orow, x, c, nx)] = __float2bfloat16(t);
      }
    }
  }
}

// The 1-channel input layer: out[v][co] = act(sum_tap in[v+off] W[tap][co] + b[co]).
// A thread forms V voxels consecutive in x (nx a multiple of V): per (dz, dy)
// line it loads the V+2 inputs once, and each tap's 16 weights (shared memory)
// once for all V voxels; two 16-byte BF16 stores per voxel.
template <int V>
__device__ __forceinline__ void conv3_in1_body(const float *in, const float *W, const float *bias,
                                               __nv_bfloat16 *out, int nx, int ny, int nz, int nb, int relu) {
  __shared__ __align__(16) float sw[27 * 16 + 16];
  for (int e = threadIdx.x; e < 27 * 16 + 16; e += blockDim.x) sw[e] = e < 27 * 16 ? W[e] : bias[e - 27 * 16];
  __syncthreads();
  const int64_t ngroups = (int64_t)nx * ny * nz * nb / V;
  for (int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gi < ngroups;
       gi += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v0 = gi * V;
    const int64_t row = v0 / nx;  // (b, z, y)
    const int x0 = (int)(v0 - row * nx), y = (int)(row % ny), z = (int)((row / ny) % nz);
    float acc[V][16];
#pragma unroll
    for (int j = 0; j < V; ++j)
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[j][c] = sw[27 * 16 + c];
    // the nine (dz, dy) lines in turn; line li+1 is loaded while line li is used
    float s[2][V + 2];
    auto load_line = [&](int li, float *dst) {
      const int dz = li / 3 - 1, dy = li % 3 - 1;
      const bool line = (unsigned)(y + dy) < (unsigned)ny && (unsigned)(z + dz) < (unsigned)nz;
      const float *p = in + v0 + (int64_t)dy * nx + (int64_t)dz * nx * ny;
#pragma unroll
      for (int k = 0; k < V + 2; ++k) {
        const int xx = x0 + k - 1;
        dst[k] = (line && (unsigned)xx < (unsigned)nx) ? __ldg(p + k - 1) : 0.f;
      }
    };
    load_line(0, s[0]);
#pragma unroll
    for (int li = 0; li < 9; ++li) {
      if (li + 1 < 9) load_line(li + 1, s[(li + 1) & 1]);
      const float *sl = s[li & 1];
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const float4 *w4 = reinterpret_cast<const float4 *>(sw + (li * 3 + (dx + 1)) * 16);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 w = w4[q];
#pragma unroll
          for (int j = 0; j < V; ++j) {
            const float a = sl[j + dx + 1];
            acc[j][4 * q] = fmaf(a, w.x, acc[j][4 * q]);
            acc[j][4 * q + 1] = fmaf(a, w.y, acc[j][4 * q + 1]);
            acc[j][4 * q + 2] = fmaf(a, w.z, acc[j][4 * q + 2]);
            acc[j][4 * q + 3] = fmaf(a, w.w, acc[j][4 * q + 3]);
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < V; ++j) {
      uint32_t w[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        float lo = acc[j][2 * c], hi = acc[j][2 * c + 1];
        if (relu) {
          lo = fmaxf(lo, 0.f);
          hi = fmaxf(hi, 0.f);
        }
        const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        w[c] = *reinterpret_cast<const uint32_t *>(&h);
      }
      *reinterpret_cast<uint4 *>(out + act_unit(row, 0, x0 + j, nx) * 8) = make_uint4(w[0], w[1], w[2], w[3]);
      *reinterpret_cast<uint4 *>(out + act_unit(row, 1, x0 + j, nx) * 8) = make_uint4(w[4], w[5], w[6], w[7]);
    }
  }
}
__global__ void __launch_bounds__(256) k_conv3_in1(const float *in, const float *W, const float *bias,
                                                   __nv_bfloat16 *out, int nx, int ny, int nz, int nb, int relu) {
  conv3_in1_body<1>(in, W, bias, out, nx, ny, nz, nb, relu);
}
__global__ void __launch_bounds__(256, 2) k_conv3_in1x4(const float *in, const float *W, const float *bias,
                                                     __nv_bfloat16 *out, int nx, int ny, int nz, int nb, int relu) {
  conv3_in1_body<4>(in, W, bias, out, nx, ny, nz, nb, relu);
}

// ---- resampling (row-planar 16-channel tensors; fine dims nx, ny, nz even) -------------------
// Decomposes a unit index of a row-planar tensor into (row, half, x).  Indices
// below 2^32 (every grid of fewer than 2^31 voxels) divide in 32 bits, several
// times cheaper than the 64-bit division.
__device__ __forceinline__ void unit_coords(int64_t u, int nx, int64_t *row, int *h, int *x) {
  if ((uint64_t)u <= 0xFFFFFFFFull) {
    const uint32_t uu = (uint32_t)u, t = uu / (uint32_t)nx;
    *x = (int)(uu - t * (uint32_t)nx);
    *h = (int)(t & 1u);
    *row = (int64_t)(t >> 1);
    return;
  }
  *x = (int)(u % nx);
  const int64_t t = u / nx;
  *h = (int)(t & 1);
  *row = t >> 1;
}
// Row index of (b, z, y) and its inverse.
__device__ __forceinline__ void row_coords(int64_t row, int ny, int nz, int64_t *b, int *z, int *y) {
  if ((uint64_t)row <= 0xFFFFFFFFull) {
    const uint32_t r = (uint32_t)row, t = r / (uint32_t)ny, bb = t / (uint32_t)nz;
    *y = (int)(r - t * (uint32_t)ny);
    *z = (int)(t - bb * (uint32_t)nz);
    *b = (int64_t)bb;
    return;
  }
  *y = (int)(row % ny);
  const int64_t t = row / ny;
  *z = (int)(t % nz);
  *b = t / nz;
}

// 2x2x2 average pooling, one thread per coarse 16-byte unit (8 channels).
__global__ void k_pool(const __nv_bfloat16 *in, __nv_bfloat16 *out, int nx, int ny, int nz, int nb) {
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
  const int64_t n = (int64_t)cx * cy * cz * nb * 2;
  const uint4 *src = reinterpret_cast<const uint4 *>(in);
  uint4 *dst = reinterpret_cast<uint4 *>(out);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t row, b;
    int h, xc, zc, yc;
    unit_coords(e, cx, &row, &h, &xc);
    row_coords(row, cy, cz, &b, &zc, &yc);
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < 8; ++k) {
      const int64_t rf = (b * nz + 2 * zc + (k >> 2)) * ny + 2 * yc + ((k >> 1) & 1);
      const uint4 q = src[act_unit(rf, h, 2 * xc + (k & 1), nx)];
      const __nv_bfloat162 *p2 = reinterpret_cast<const __nv_bfloat162 *>(&q);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float2 f = __bfloat1622float2(p2[c]);
        s[2 * c] += f.x;
        s[2 * c + 1] += f.y;
      }
    }
    uint4 o;
    __nv_bfloat162 *o2 = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
    for (int c = 0; c < 4; ++c) o2[c] = __floats2bfloat162_rn(0.125f * s[2 * c], 0.125f * s[2 * c + 1]);
    dst[e] = o;
  }
}
// Nearest-neighbour 2x upsampling: fine (nx,ny,nz) from coarse (nx/2,...).  One
// thread per coarse 16-byte unit: one load, and its eight fine copies as two
// adjacent units in each of the four fine rows (a warp writes 1 KB runs).
__global__ void k_upsample(const __nv_bfloat16 *in, __nv_bfloat16 *out, int nx, int ny, int nz, int nb) {
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
  const int64_t n = (int64_t)cx * cy * cz * nb * 2;
  const uint4 *src = reinterpret_cast<const uint4 *>(in);
  uint4 *dst = reinterpret_cast<uint4 *>(out);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t row, b;
    int h, xc, zc, yc;
    unit_coords(e, cx, &row, &h, &xc);
    row_coords(row, cy, cz, &b, &zc, &yc);
    const uint4 v = src[e];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t rf = (b * nz + 2 * zc + (k >> 1)) * ny + 2 * yc + (k & 1);
      uint4 *d = dst + act_unit(rf, h, 2 * xc, nx);
      d[0] = v;
      d[1] = v;
    }
  }
}
// Backward of pooling: d_fine += d_coarse / 8 (FP32 row-planar tensors).
__global__ void k_pool_bwd(const float *dc, float *df, int nx, int ny, int nz, int nb) {
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
  const int64_t n = (int64_t)nx * ny * nz * nb * 16;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t row, b;
    int h, x, z, y;
    unit_coords(e >> 3, nx, &row, &h, &x);
    row_coords(row, ny, nz, &b, &z, &y);
    df[e] += 0.125f * dc[act_unit((b * cz + z / 2) * cy + y / 2, h, x / 2, cx) * 8 + (e & 7)];
  }
}
// Backward of nearest upsampling: d_coarse = sum of the 8 fine children.
__global__ void k_up_bwd(const float *df, float *dc, int nx, int ny, int nz, int nb) {
  const int cx = nx / 2, cy = ny / 2, cz = nz / 2;
  const int64_t n = (int64_t)cx * cy * cz * nb * 16;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t row, b;
    int h, xc, zc, yc;
    unit_coords(e >> 3, cx, &row, &h, &xc);
    row_coords(row, cy, cz, &b, &zc, &yc);
    float s = 0.f;
    for (int k = 0; k < 8; ++k) {
      const int64_t rf = (b * nz + 2 * zc + (k >> 2)) * ny + 2 * yc + ((k >> 1) & 1);
      s += df[act_unit(rf, h, 2 * xc + (k & 1), nx) * 8 + (e & 7)];
    }
    dc[e] = s;
  }
}
// dpre = d * (act > 0), to BF16 (the next backward conv's input) and optionally FP32.
__global__ void k_relu_mask(const float *d, const __nv_bfloat16 *act, __nv_bfloat16 *out, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = __float2bfloat16(__bfloat162float(act[e]) > 0.f ? d[e] : 0.f);
}
__global__ void k_add_f32(const float *src, float *dst, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    dst[e] += src[e];
}

// ---- gradients --------------------------------------------------------------------------------
// Per block partial of dW[tap][ci][co] = sum_v X[v+off(tap)][ci] dY[v][co] and
// dbias[co] = sum_v dY[v][co] over the voxels v = blockIdx.x, +gridDim.x, ...
// Task t < 27*cin is (tap, ci); task 27*cin is the bias.  partial layout:
// [block][27*cin + 1][16].  A fixed grid and a fixed block-order reduction
// (k_reduce_partials) keep the gradients deterministic.
__global__ void __launch_bounds__(256) k_dW(DwArgs a) {
  const int ntask = 27 * a.cin + 1;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int64_t nvox = (int64_t)nx * ny * nz * a.nb;
  __shared__ float sdy[64][16];
  for (int task0 = 0; task0 < ntask; task0 += blockDim.x) {
    const int task = task0 + threadIdx.x;
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c] = 0.f;
    const int tap = task < 27 * a.cin ? task / a.cin : 0, ci = task < 27 * a.cin ? task % a.cin : 0;
    const int ox = tap % 3 - 1, oy = (tap / 3) % 3 - 1, oz = tap / 9 - 1;
    for (int64_t v0 = (int64_t)blockIdx.x * 64; v0 < nvox; v0 += (int64_t)gridDim.x * 64) {
      __syncthreads();
      for (int e = threadIdx.x; e < 64 * 16; e += blockDim.x) {
        const int64_t v = v0 + e / 16;
        sdy[e / 16][e % 16] = v < nvox ? __bfloat162float(a.dy[act_elem(v / nx, (int)(v % nx), e % 16, nx)]) : 0.f;
      }
      __syncthreads();
      if (task >= ntask) continue;
      for (int j = 0; j < 64 && v0 + j < nvox; ++j) {
        const int64_t v = v0 + j;
        float s = 1.f;
        if (task < 27 * a.cin) {
          const int x = (int)(v % nx) + ox, y = (int)((v / nx) % ny) + oy, z = (int)((v / ((int64_t)nx * ny)) % nz) + oz;
          if (x < 0 || x >= nx || y < 0 || y >= ny || z < 0 || z >= nz) continue;
          const int64_t b = v / ((int64_t)nx * ny * nz);
          const int64_t row = (b * nz + z) * ny + y;
          if (a.x_f32) s = a.x_f32[row * nx + x];
          else s = __bfloat162float(ci < 16 ? a.x0[act_elem(row, x, ci, nx)] : a.x1[act_elem(row, x, ci - 16, nx)]);
        }
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = fmaf(s, sdy[j][c], acc[c]);
      }
    }
    if (task < ntask) {
      float *o = a.partial + ((size_t)blockIdx.x * ntask + task) * 16;
#pragma unroll
      for (int c = 0; c < 16; ++c) o[c] = acc[c];
    }
  }
}
// grad[k] (+)= sum over blocks of partial[block][k], k < n, in block order.
__global__ void k_reduce_partials(const float *partial, int nblocks, int n, float *grad, int accumulate) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * n + k];
    grad[k] = accumulate ? grad[k] + s : s;
  }
}

// Output projection (training path): out[v] = proj . act[v] + proj_b.
__global__ void k_proj_fwd(const __nv_bfloat16 *act, const float *proj, float *out, int64_t nvox, int nx) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
    float r = proj[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) r = fmaf(proj[c], __bfloat162float(act[act_elem(v / nx, (int)(v % nx), c, nx)]), r);
    out[v] = r;
  }
}
// d act = proj * dOut (masked by act > 0, to BF16); per-block partials of
// dproj[c] = sum act[v][c] dOut[v] and dproj_b = sum dOut[v] ([block][17]).
__global__ void __launch_bounds__(256) k_proj_bwd(const __nv_bfloat16 *act, const float *proj, const float *dout,
                                                  __nv_bfloat16 *dact, float *partial, int64_t nvox, int nx) {
  __shared__ float red[17][256];
  float acc[17];
#pragma unroll
  for (int c = 0; c < 17; ++c) acc[c] = 0.f;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
    const float d = dout[v];
    const int64_t row = v / nx;
    const int x = (int)(v % nx);
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int64_t e = act_elem(row, x, c, nx);
      const float av = __bfloat162float(act[e]);
      acc[c] = fmaf(av, d, acc[c]);
      dact[e] = __float2bfloat16(av > 0.f ? proj[c] * d : 0.f);
    }
    acc[16] += d;
  }
#pragma unroll
  for (int c = 0; c < 17; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 17; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 17) partial[(size_t)blockIdx.x * 17 + threadIdx.x] = red[threadIdx.x][0];
}

// Mean squared error over n values and dL/dout; per-block loss partials.
__global__ void __launch_bounds__(256) k_mse(const float *out, const float *tgt, float *dout, float *partial,
                                             int64_t n) {
  __shared__ float red[256];
  float s = 0.f;
  const float scale = 2.f / (float)n;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const float e = out[v] - tgt[v];
    s += e * e;
    dout[v] = scale * e;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Energy-norm loss of the HPCCG operator A (the 27-point generate_matrix
// stencil: 27 on the diagonal, -1 for each neighbour inside the grid):
// L = (1/n) d.(A d), d = target - out, per grid of the batch; dL/dout = -(2/n) A d.
__global__ void __launch_bounds__(256) k_energy(const float *out, const float *tgt, float *dout, float *partial,
                                                int nx, int ny, int nz, int nb) {
  __shared__ float red[256];
  const int64_t n = (int64_t)nx * ny * nz * nb;
  const float scale = 2.f / (float)n;
  float s = 0.f;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)((v / ((int64_t)nx * ny)) % nz);
    const int64_t b = v / ((int64_t)nx * ny * nz);
    float ad = 0.f;
    for (int t = 0; t < 27; ++t) {
      const int xx = x + t % 3 - 1, yy = y + (t / 3) % 3 - 1, zz = z + t / 9 - 1;
      if (xx < 0 || xx >= nx || yy < 0 || yy >= ny || zz < 0 || zz >= nz) continue;
      const int64_t u = ((b * nz + zz) * ny + yy) * nx + xx;
      const float du = tgt[u] - out[u];
      ad += (t == 13 ? 27.f : -1.f) * du;
    }
    s += (tgt[v] - out[v]) * ad;
    dout[v] = -scale * ad;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
  }
}

}  // namespace hpccg
