// unet.cu -- the learned preconditioner: a 4-level 3D U-Net, 16 channels at
// every level (104,337 parameters), BF16 activations, FP32 accumulation and
// FP32 master weights, trained and applied with this project's own kernels.
//
//   level 0 (n)   : e1a = relu(conv(r; 1->16))   e1b = relu(conv(e1a))
//   level 1 (n/2) : e2a, e2b on pool(e1b)        (2x2x2 average pooling)
//   level 2 (n/4) : e3a, e3b on pool(e2b)
//   level 3 (n/8) : e4a, e4b on pool(e3b)
//   decoder       : c3a = relu(conv(e3b ++ up(e4b))), c3b;  c2a(e2b ++ up(c3b)), c2b;
//                   out = proj . relu(conv(e1b ++ up(c2b))) + b  (1 channel, FP32)
// "++" is a virtual concatenation: the conv reads both 16-channel tensors.
// 16-channel convs on volumes of >= 128 voxels run on tcgen05 (unet_conv.cu),
// the 1-channel input conv and smaller volumes on CUDA cores (unet_ops.cu).
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "unet_ops.cuh"

namespace hpccg {

struct LayerDef {
  int cin, nin, level;
};
// Layers in parameter order; nin = number of 16-channel BF16 input groups (0 = the FP32 input).
static const LayerDef kLayers[13] = {{1, 0, 0},  {16, 1, 0}, {16, 1, 1}, {16, 1, 1}, {16, 1, 2},
                                     {16, 1, 2}, {16, 1, 3}, {16, 1, 3}, {32, 2, 2}, {16, 1, 2},
                                     {32, 2, 1}, {16, 1, 1}, {32, 2, 0}};
constexpr int kNumLayers = 13;

struct Level {
  int nx = 0, ny = 0, nz = 0;
  int64_t nvox = 0;  // including the batch
};

}  // namespace hpccg

using namespace hpccg;

struct hpccg_unet {
  int device = 0, num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int nparams = 0;
  int off[kNumLayers + 1] = {};  // layer parameter offsets; off[13] = projection
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  int adam_t = 0;
  __nv_bfloat16 *packed_fwd[kNumLayers] = {}, *packed_bwd[kNumLayers][2] = {};
  float *flip[kNumLayers][2] = {};  // FP32 flipped weights for CUDA-core backward-data
  float *partial = nullptr;         // gradient partials
  int partial_blocks = 0;
  int *d_err = nullptr;
  // activations for the current shape
  int nx = 0, ny = 0, nz = 0, nb = 0;
  bool train_bufs = false;
  Level L[4];
  __nv_bfloat16 *e1a = nullptr, *e1b = nullptr, *u1 = nullptr, *c1 = nullptr;
  __nv_bfloat16 *d1 = nullptr, *e2a = nullptr, *e2b = nullptr, *u2 = nullptr, *c2a = nullptr, *c2b = nullptr;
  __nv_bfloat16 *d2 = nullptr, *e3a = nullptr, *e3b = nullptr, *u3 = nullptr, *c3a = nullptr, *c3b = nullptr;
  __nv_bfloat16 *d3 = nullptr, *e4a = nullptr, *e4b = nullptr;
  // backward buffers (FP32 gradients per level, BF16 masked pre-activation gradients)
  float *g[4] = {}, *gs[4] = {}, *gt[4] = {};
  __nv_bfloat16 *pre[4] = {};
  float *out_train = nullptr, *dout = nullptr;
  int loss_kind = 0;  // 0 = mean squared error, 1 = energy norm of the HPCCG operator
  std::vector<void *> act_allocs;
};

namespace hpccg {

static int grid1d(const hpccg_unet *u, int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)u->num_sms * 16));
}

static void free_acts(hpccg_unet *u) {
  for (void *p : u->act_allocs) cudaFree(p);
  u->act_allocs.clear();
  u->nx = u->ny = u->nz = u->nb = 0;
  u->train_bufs = false;
}

template <typename T>
static int alloc_act(hpccg_unet *u, T **p, int64_t count) {
  HPCCG_CUDA(cudaMalloc(p, sizeof(T) * std::max<int64_t>(count, 1)));
  u->act_allocs.push_back(*p);
  return HPCCG_OK;
}

// Activation (and, for training, gradient) buffers for one input shape.
static int ensure_shape(hpccg_unet *u, int nx, int ny, int nz, int nb, bool train) {
  if (nx % 8 || ny % 8 || nz % 8 || nx < 8 || ny < 8 || nz < 8 || nb < 1) return HPCCG_ERR_INVALID_ARG;
  if (u->nx == nx && u->ny == ny && u->nz == nz && u->nb == nb && (u->train_bufs || !train)) return HPCCG_OK;
  free_acts(u);
  for (int l = 0; l < 4; ++l) {
    u->L[l].nx = nx >> l;
    u->L[l].ny = ny >> l;
    u->L[l].nz = nz >> l;
    u->L[l].nvox = (int64_t)u->L[l].nx * u->L[l].ny * u->L[l].nz * nb;
  }
  const int64_t c0 = u->L[0].nvox * 16, c1 = u->L[1].nvox * 16, c2 = u->L[2].nvox * 16, c3 = u->L[3].nvox * 16;
  int rc = 0;
  __nv_bfloat16 **b0[] = {&u->e1a, &u->e1b, &u->u1};
  for (auto p : b0) if ((rc = alloc_act(u, p, c0))) return rc;
  __nv_bfloat16 **b1[] = {&u->d1, &u->e2a, &u->e2b, &u->u2, &u->c2a, &u->c2b};
  for (auto p : b1) if ((rc = alloc_act(u, p, c1))) return rc;
  __nv_bfloat16 **b2[] = {&u->d2, &u->e3a, &u->e3b, &u->u3, &u->c3a, &u->c3b};
  for (auto p : b2) if ((rc = alloc_act(u, p, c2))) return rc;
  __nv_bfloat16 **b3[] = {&u->d3, &u->e4a, &u->e4b};
  for (auto p : b3) if ((rc = alloc_act(u, p, c3))) return rc;
  if (train) {
    if ((rc = alloc_act(u, &u->c1, c0))) return rc;
    for (int l = 0; l < 4; ++l) {
      const int64_t c = u->L[l].nvox * 16;
      if ((rc = alloc_act(u, &u->g[l], c))) return rc;
      if ((rc = alloc_act(u, &u->gs[l], c))) return rc;
      if ((rc = alloc_act(u, &u->gt[l], c))) return rc;
      if ((rc = alloc_act(u, &u->pre[l], c))) return rc;
    }
    if ((rc = alloc_act(u, &u->out_train, u->L[0].nvox))) return rc;
    if ((rc = alloc_act(u, &u->dout, u->L[0].nvox))) return rc;
    u->train_bufs = true;
  }
  u->nx = nx;
  u->ny = ny;
  u->nz = nz;
  u->nb = nb;
  return HPCCG_OK;
}

static int repack(hpccg_unet *u) {
  for (int l = 0; l < kNumLayers; ++l) {
    const LayerDef &d = kLayers[l];
    const float *W = u->params + u->off[l];
    if (d.nin > 0) {
      k_pack_fwd<<<32, 256, 0, u->stream>>>(W, d.cin, d.nin, u->packed_fwd[l]);
      for (int gi = 0; gi < d.nin; ++gi) {
        k_pack_bwd<<<32, 256, 0, u->stream>>>(W, d.cin, gi, u->packed_bwd[l][gi]);
        k_flip_fp32<<<32, 256, 0, u->stream>>>(W, d.cin, gi, u->flip[l][gi]);
      }
    }
  }
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

// One 16-output conv: tcgen05 when the level holds whole 128-voxel bricks,
// CUDA cores otherwise.  `bwd_group` >= 0 selects the backward-data conv of
// that input group (input in0 = the 16-channel pre-activation gradient).
static int conv(hpccg_unet *u, int layer, int level, const __nv_bfloat16 *in0, const __nv_bfloat16 *in1,
                const float *in_f32, int epi, void *out, int bwd_group = -1) {
  const LayerDef &d = kLayers[layer];
  const Level &Lv = u->L[level];
  const float *W = u->params + u->off[layer];
  const float *bias = W + 27 * d.cin * 16;
  const float *proj = u->params + u->off[kNumLayers];
  const int nin = bwd_group >= 0 ? 1 : d.nin;
  ConvGeom g;
  if (nin > 0 && conv_geom(Lv.nx, Lv.ny, Lv.nz, u->nb, &g)) {
    ConvArgs a;
    a.g = g;
    a.in0 = in0;
    a.in1 = in1;
    a.wpack = bwd_group >= 0 ? u->packed_bwd[layer][bwd_group] : u->packed_fwd[layer];
    a.bias = bwd_group >= 0 ? nullptr : bias;
    a.proj = proj;
    a.out = out;
    a.err = u->d_err;
    return launch_conv3_tc(nin, epi, a, u->num_sms, u->stream);
  }
  if (in_f32 && (epi == kEpiBiasRelu || epi == kEpiBias)) {  // the 1-channel input layer
    if (Lv.nx % 128 == 0)  // tensor cores, 128-voxel row tiles
      return launch_conv3_in1_tc(in_f32, W, bias, static_cast<__nv_bfloat16 *>(out), Lv.nx, Lv.ny, Lv.nz, u->nb,
                                 epi == kEpiBiasRelu, u->d_err, u->num_sms, u->stream);
    if (Lv.nx % 4 == 0)
      k_conv3_in1x4<<<grid1d(u, Lv.nvox / 4), 256, 0, u->stream>>>(
          in_f32, W, bias, static_cast<__nv_bfloat16 *>(out), Lv.nx, Lv.ny, Lv.nz, u->nb, epi == kEpiBiasRelu);
    else
      k_conv3_in1<<<grid1d(u, Lv.nvox), 256, 0, u->stream>>>(
          in_f32, W, bias, static_cast<__nv_bfloat16 *>(out), Lv.nx, Lv.ny, Lv.nz, u->nb, epi == kEpiBiasRelu);
    HPCCG_CUDA(cudaGetLastError());
    return HPCCG_OK;
  }
  CcConvArgs a;
  a.nx = Lv.nx;
  a.ny = Lv.ny;
  a.nz = Lv.nz;
  a.nb = u->nb;
  a.nin = nin;
  a.cin = bwd_group >= 0 ? 16 : d.cin;
  a.in0 = in0;
  a.in1 = in1;
  a.in_f32 = in_f32;
  a.W = bwd_group >= 0 ? u->flip[layer][bwd_group] : W;
  a.bias = bwd_group >= 0 ? nullptr : bias;
  a.proj = proj;
  a.epi = epi;
  a.out = out;
  k_conv3_cc<<<grid1d(u, Lv.nvox), 256, 0, u->stream>>>(a);
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

#define UNET_TRY(x)              \
  do {                           \
    const int rc_ = (x);         \
    if (rc_) return rc_;         \
  } while (0)

// Forward pass.  train: store c1 and write the projection to u->out_train.
static int forward(hpccg_unet *u, const float *in, float *out, bool train) {
  const Level *L = u->L;
  UNET_TRY(conv(u, 0, 0, nullptr, nullptr, in, kEpiBiasRelu, u->e1a));
  UNET_TRY(conv(u, 1, 0, u->e1a, nullptr, nullptr, kEpiBiasRelu, u->e1b));
  k_pool<<<grid1d(u, L[1].nvox * 2), 256, 0, u->stream>>>(u->e1b, u->d1, L[0].nx, L[0].ny, L[0].nz, u->nb);
  UNET_TRY(conv(u, 2, 1, u->d1, nullptr, nullptr, kEpiBiasRelu, u->e2a));
  UNET_TRY(conv(u, 3, 1, u->e2a, nullptr, nullptr, kEpiBiasRelu, u->e2b));
  k_pool<<<grid1d(u, L[2].nvox * 2), 256, 0, u->stream>>>(u->e2b, u->d2, L[1].nx, L[1].ny, L[1].nz, u->nb);
  UNET_TRY(conv(u, 4, 2, u->d2, nullptr, nullptr, kEpiBiasRelu, u->e3a));
  UNET_TRY(conv(u, 5, 2, u->e3a, nullptr, nullptr, kEpiBiasRelu, u->e3b));
  k_pool<<<grid1d(u, L[3].nvox * 2), 256, 0, u->stream>>>(u->e3b, u->d3, L[2].nx, L[2].ny, L[2].nz, u->nb);
  UNET_TRY(conv(u, 6, 3, u->d3, nullptr, nullptr, kEpiBiasRelu, u->e4a));
  UNET_TRY(conv(u, 7, 3, u->e4a, nullptr, nullptr, kEpiBiasRelu, u->e4b));
  k_upsample<<<grid1d(u, L[2].nvox / 4), 256, 0, u->stream>>>(u->e4b, u->u3, L[2].nx, L[2].ny, L[2].nz, u->nb);
  UNET_TRY(conv(u, 8, 2, u->e3b, u->u3, nullptr, kEpiBiasRelu, u->c3a));
  UNET_TRY(conv(u, 9, 2, u->c3a, nullptr, nullptr, kEpiBiasRelu, u->c3b));
  k_upsample<<<grid1d(u, L[1].nvox / 4), 256, 0, u->stream>>>(u->c3b, u->u2, L[1].nx, L[1].ny, L[1].nz, u->nb);
  UNET_TRY(conv(u, 10, 1, u->e2b, u->u2, nullptr, kEpiBiasRelu, u->c2a));
  UNET_TRY(conv(u, 11, 1, u->c2a, nullptr, nullptr, kEpiBiasRelu, u->c2b));
  k_upsample<<<grid1d(u, L[0].nvox / 4), 256, 0, u->stream>>>(u->c2b, u->u1, L[0].nx, L[0].ny, L[0].nz, u->nb);
  if (train) {
    UNET_TRY(conv(u, 12, 0, u->e1b, u->u1, nullptr, kEpiBiasRelu, u->c1));
    k_proj_fwd<<<grid1d(u, L[0].nvox), 256, 0, u->stream>>>(u->c1, u->params + u->off[kNumLayers], out, L[0].nvox,
                                                           L[0].nx);
  } else {
    UNET_TRY(conv(u, 12, 0, u->e1b, u->u1, nullptr, kEpiProject, out));
  }
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

// Weight/bias gradient of `layer` from its forward inputs and the masked
// pre-activation gradient dy (BF16), accumulated into u->grads.
static int weight_grad(hpccg_unet *u, int layer, int level, const __nv_bfloat16 *x0, const __nv_bfloat16 *x1,
                       const float *xf, const __nv_bfloat16 *dy) {
  const LayerDef &d = kLayers[layer];
  DwArgs a;
  a.nx = u->L[level].nx;
  a.ny = u->L[level].ny;
  a.nz = u->L[level].nz;
  a.nb = u->nb;
  a.cin = d.cin;
  a.x0 = x0;
  a.x1 = x1;
  a.x_f32 = xf;
  a.dy = dy;
  a.partial = u->partial;
  const int blocks = (int)std::min<int64_t>(u->partial_blocks, (u->L[level].nvox + 63) / 64);
  k_dW<<<blocks, 256, 0, u->stream>>>(a);
  const int n = (27 * d.cin + 1) * 16;
  k_reduce_partials<<<(n + 255) / 256, 256, 0, u->stream>>>(u->partial, blocks, n, u->grads + u->off[layer], 1);
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

static void mask(hpccg_unet *u, int level, const float *gsrc, const __nv_bfloat16 *act, __nv_bfloat16 *dst) {
  const int64_t n = u->L[level].nvox * 16;
  k_relu_mask<<<grid1d(u, n), 256, 0, u->stream>>>(gsrc, act, dst, n);
}

// Backward pass from u->dout (dL/dout), accumulating into u->grads.
static int backward(hpccg_unet *u, const float *in) {
  const Level *L = u->L;
  const int nb = u->nb;
  cudaStream_t s = u->stream;
  // projection and dec1a (level 0)
  const int pb = (int)std::min<int64_t>(u->partial_blocks, (L[0].nvox + 255) / 256);
  k_proj_bwd<<<pb, 256, 0, s>>>(u->c1, u->params + u->off[kNumLayers], u->dout, u->pre[0], u->partial, L[0].nvox,
                                L[0].nx);
  k_reduce_partials<<<1, 32, 0, s>>>(u->partial, pb, 17, u->grads + u->off[kNumLayers], 1);
  UNET_TRY(weight_grad(u, 12, 0, u->e1b, u->u1, nullptr, u->pre[0]));
  UNET_TRY(conv(u, 12, 0, u->pre[0], nullptr, nullptr, kEpiRawF32, u->gs[0], 0));  // d e1b (skip)
  UNET_TRY(conv(u, 12, 0, u->pre[0], nullptr, nullptr, kEpiRawF32, u->gt[0], 1));  // d u1
  k_up_bwd<<<grid1d(u, L[1].nvox * 16), 256, 0, s>>>(u->gt[0], u->g[1], L[0].nx, L[0].ny, L[0].nz, nb);
  // dec2b, dec2a (level 1)
  mask(u, 1, u->g[1], u->c2b, u->pre[1]);
  UNET_TRY(weight_grad(u, 11, 1, u->c2a, nullptr, nullptr, u->pre[1]));
  UNET_TRY(conv(u, 11, 1, u->pre[1], nullptr, nullptr, kEpiRawF32, u->g[1], 0));
  mask(u, 1, u->g[1], u->c2a, u->pre[1]);
  UNET_TRY(weight_grad(u, 10, 1, u->e2b, u->u2, nullptr, u->pre[1]));
  UNET_TRY(conv(u, 10, 1, u->pre[1], nullptr, nullptr, kEpiRawF32, u->gs[1], 0));  // d e2b (skip)
  UNET_TRY(conv(u, 10, 1, u->pre[1], nullptr, nullptr, kEpiRawF32, u->gt[1], 1));  // d u2
  k_up_bwd<<<grid1d(u, L[2].nvox * 16), 256, 0, s>>>(u->gt[1], u->g[2], L[1].nx, L[1].ny, L[1].nz, nb);
  // dec3b, dec3a (level 2)
  mask(u, 2, u->g[2], u->c3b, u->pre[2]);
  UNET_TRY(weight_grad(u, 9, 2, u->c3a, nullptr, nullptr, u->pre[2]));
  UNET_TRY(conv(u, 9, 2, u->pre[2], nullptr, nullptr, kEpiRawF32, u->g[2], 0));
  mask(u, 2, u->g[2], u->c3a, u->pre[2]);
  UNET_TRY(weight_grad(u, 8, 2, u->e3b, u->u3, nullptr, u->pre[2]));
  UNET_TRY(conv(u, 8, 2, u->pre[2], nullptr, nullptr, kEpiRawF32, u->gs[2], 0));  // d e3b (skip)
  UNET_TRY(conv(u, 8, 2, u->pre[2], nullptr, nullptr, kEpiRawF32, u->gt[2], 1));  // d u3
  k_up_bwd<<<grid1d(u, L[3].nvox * 16), 256, 0, s>>>(u->gt[2], u->g[3], L[2].nx, L[2].ny, L[2].nz, nb);
  // enc4b, enc4a (level 3)
  mask(u, 3, u->g[3], u->e4b, u->pre[3]);
  UNET_TRY(weight_grad(u, 7, 3, u->e4a, nullptr, nullptr, u->pre[3]));
  UNET_TRY(conv(u, 7, 3, u->pre[3], nullptr, nullptr, kEpiRawF32, u->g[3], 0));
  mask(u, 3, u->g[3], u->e4a, u->pre[3]);
  UNET_TRY(weight_grad(u, 6, 3, u->d3, nullptr, nullptr, u->pre[3]));
  UNET_TRY(conv(u, 6, 3, u->pre[3], nullptr, nullptr, kEpiRawF32, u->g[3], 0));  // d d3
  k_pool_bwd<<<grid1d(u, L[2].nvox * 16), 256, 0, s>>>(u->g[3], u->gs[2], L[2].nx, L[2].ny, L[2].nz, nb);
  // enc3b, enc3a (level 2)
  mask(u, 2, u->gs[2], u->e3b, u->pre[2]);
  UNET_TRY(weight_grad(u, 5, 2, u->e3a, nullptr, nullptr, u->pre[2]));
  UNET_TRY(conv(u, 5, 2, u->pre[2], nullptr, nullptr, kEpiRawF32, u->g[2], 0));
  mask(u, 2, u->g[2], u->e3a, u->pre[2]);
  UNET_TRY(weight_grad(u, 4, 2, u->d2, nullptr, nullptr, u->pre[2]));
  UNET_TRY(conv(u, 4, 2, u->pre[2], nullptr, nullptr, kEpiRawF32, u->g[2], 0));  // d d2
  k_pool_bwd<<<grid1d(u, L[1].nvox * 16), 256, 0, s>>>(u->g[2], u->gs[1], L[1].nx, L[1].ny, L[1].nz, nb);
  // enc2b, enc2a (level 1)
  mask(u, 1, u->gs[1], u->e2b, u->pre[1]);
  UNET_TRY(weight_grad(u, 3, 1, u->e2a, nullptr, nullptr, u->pre[1]));
  UNET_TRY(conv(u, 3, 1, u->pre[1], nullptr, nullptr, kEpiRawF32, u->g[1], 0));
  mask(u, 1, u->g[1], u->e2a, u->pre[1]);
  UNET_TRY(weight_grad(u, 2, 1, u->d1, nullptr, nullptr, u->pre[1]));
  UNET_TRY(conv(u, 2, 1, u->pre[1], nullptr, nullptr, kEpiRawF32, u->g[1], 0));  // d d1
  k_pool_bwd<<<grid1d(u, L[0].nvox * 16), 256, 0, s>>>(u->g[1], u->gs[0], L[0].nx, L[0].ny, L[0].nz, nb);
  // enc1b, enc1a (level 0)
  mask(u, 0, u->gs[0], u->e1b, u->pre[0]);
  UNET_TRY(weight_grad(u, 1, 0, u->e1a, nullptr, nullptr, u->pre[0]));
  UNET_TRY(conv(u, 1, 0, u->pre[0], nullptr, nullptr, kEpiRawF32, u->g[0], 0));
  mask(u, 0, u->g[0], u->e1a, u->pre[0]);
  UNET_TRY(weight_grad(u, 0, 0, nullptr, nullptr, in, u->pre[0]));
  HPCCG_CUDA(cudaGetLastError());
  return HPCCG_OK;
}

static int check_err(hpccg_unet *u) {
  int err = 0;
  HPCCG_CUDA(cudaMemcpyAsync(&err, u->d_err, sizeof(int), cudaMemcpyDeviceToHost, u->stream));
  HPCCG_CUDA(cudaStreamSynchronize(u->stream));
  if (err) {
    cudaMemsetAsync(u->d_err, 0, sizeof(int), u->stream);
    cudaStreamSynchronize(u->stream);
    return HPCCG_ERR_TIMEOUT;
  }
  return HPCCG_OK;
}

// splitmix64 uniform in [-1,1), the project's counter-based generator.
static double u_pm1(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return 2.0 * ((double)(z >> 11) * 0x1.0p-53) - 1.0;
}

}  // namespace hpccg

// ---------------------------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------------------------

extern "C" void hpccg_unet_destroy(hpccg_unet *u) {
  if (!u) return;
  free_acts(u);
  void *bufs[] = {u->params, u->grads, u->adam_m, u->adam_v, u->partial, u->d_err};
  for (void *p : bufs)
    if (p) cudaFree(p);
  for (int l = 0; l < kNumLayers; ++l) {
    if (u->packed_fwd[l]) cudaFree(u->packed_fwd[l]);
    for (int gi = 0; gi < 2; ++gi) {
      if (u->packed_bwd[l][gi]) cudaFree(u->packed_bwd[l][gi]);
      if (u->flip[l][gi]) cudaFree(u->flip[l][gi]);
    }
  }
  if (u->ev0) cudaEventDestroy(u->ev0);
  if (u->ev1) cudaEventDestroy(u->ev1);
  if (u->stream) cudaStreamDestroy(u->stream);
  delete u;
}

extern "C" int hpccg_unet_create(uint64_t seed, hpccg_unet **out) {
  if (!out) return HPCCG_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HPCCG_ERR_NO_DEVICE;
  hpccg_unet *u = new hpccg_unet();
  auto fail = [&](int rc) {
    hpccg_unet_destroy(u);
    return rc;
  };
  if (cudaGetDevice(&u->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&u->num_sms, cudaDevAttrMultiProcessorCount, u->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&u->ev0) != cudaSuccess || cudaEventCreate(&u->ev1) != cudaSuccess)
    return fail(HPCCG_ERR_CUDA);
  int off = 0;
  for (int l = 0; l < kNumLayers; ++l) {
    u->off[l] = off;
    off += 27 * kLayers[l].cin * 16 + 16;
  }
  u->off[kNumLayers] = off;
  off += 17;
  u->nparams = off;
  // He-uniform weights, zero biases; the projection starts small.
  std::vector<float> h(off, 0.f);
  uint64_t k = 0;
  for (int l = 0; l < kNumLayers; ++l) {
    const int fan_in = 27 * kLayers[l].cin;
    const double bound = sqrt(6.0 / fan_in);
    for (int e = 0; e < fan_in * 16; ++e) h[u->off[l] + e] = (float)(bound * u_pm1(seed, k++));
  }
  for (int c = 0; c < 16; ++c) h[u->off[kNumLayers] + c] = (float)(0.1 * sqrt(6.0 / 16) * u_pm1(seed, k++));
  const size_t pbytes = sizeof(float) * off;
  if (cudaMalloc(&u->params, pbytes) || cudaMalloc(&u->grads, pbytes) || cudaMalloc(&u->adam_m, pbytes) ||
      cudaMalloc(&u->adam_v, pbytes) || cudaMalloc(&u->d_err, sizeof(int)))
    return fail(HPCCG_ERR_OOM);
  cudaMemcpyAsync(u->params, h.data(), pbytes, cudaMemcpyHostToDevice, u->stream);
  cudaMemsetAsync(u->grads, 0, pbytes, u->stream);
  cudaMemsetAsync(u->adam_m, 0, pbytes, u->stream);
  cudaMemsetAsync(u->adam_v, 0, pbytes, u->stream);
  cudaMemsetAsync(u->d_err, 0, sizeof(int), u->stream);
  for (int l = 0; l < kNumLayers; ++l) {
    const LayerDef &d = kLayers[l];
    if (d.nin == 0) continue;
    if (cudaMalloc(&u->packed_fwd[l], sizeof(__nv_bfloat16) * d.nin * 27 * 256)) return fail(HPCCG_ERR_OOM);
    for (int gi = 0; gi < d.nin; ++gi)
      if (cudaMalloc(&u->packed_bwd[l][gi], sizeof(__nv_bfloat16) * 27 * 256) ||
          cudaMalloc(&u->flip[l][gi], sizeof(float) * 27 * 256))
        return fail(HPCCG_ERR_OOM);
  }
  u->partial_blocks = u->num_sms * 2;
  if (cudaMalloc(&u->partial, sizeof(float) * (size_t)u->partial_blocks * (27 * 32 + 1) * 16))
    return fail(HPCCG_ERR_OOM);
  int rc = repack(u);
  if (!rc && cudaStreamSynchronize(u->stream) != cudaSuccess) rc = HPCCG_ERR_CUDA;
  if (rc) return fail(rc);
  *out = u;
  return HPCCG_OK;
}

extern "C" int hpccg_unet_num_params(const hpccg_unet *u, int64_t *n) {
  if (!u || !n) return HPCCG_ERR_INVALID_ARG;
  *n = u->nparams;
  return HPCCG_OK;
}

extern "C" int hpccg_unet_get_params(const hpccg_unet *u, float *host) {
  if (!u || !host) return HPCCG_ERR_INVALID_ARG;
  HPCCG_CUDA(cudaMemcpyAsync(host, u->params, sizeof(float) * u->nparams, cudaMemcpyDeviceToHost, u->stream));
  HPCCG_CUDA(cudaStreamSynchronize(u->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_unet_set_params(hpccg_unet *u, const float *host) {
  if (!u || !host) return HPCCG_ERR_INVALID_ARG;
  HPCCG_CUDA(cudaMemcpyAsync(u->params, host, sizeof(float) * u->nparams, cudaMemcpyHostToDevice, u->stream));
  int rc = repack(u);
  if (rc) return rc;
  HPCCG_CUDA(cudaStreamSynchronize(u->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_unet_forward(hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz, int32_t nb, const float *d_in,
                                  float *d_out) {
  if (!u || !d_in || !d_out) return HPCCG_ERR_INVALID_ARG;
  int rc = ensure_shape(u, nx, ny, nz, nb, false);
  if (rc) return rc;
  if ((rc = forward(u, d_in, d_out, false))) return rc;
  return check_err(u);
}

extern "C" int hpccg_unet_loss_grad(hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz, int32_t nb,
                                    const float *d_in, const float *d_target, float *loss, float *grad_host) {
  if (!u || !d_in || !d_target) return HPCCG_ERR_INVALID_ARG;
  int rc = ensure_shape(u, nx, ny, nz, nb, true);
  if (rc) return rc;
  HPCCG_CUDA(cudaMemsetAsync(u->grads, 0, sizeof(float) * u->nparams, u->stream));
  if ((rc = forward(u, d_in, u->out_train, true))) return rc;
  const int64_t n = u->L[0].nvox;
  const int mb = std::min(u->partial_blocks, grid1d(u, n));
  if (u->loss_kind == 1)
    k_energy<<<mb, 256, 0, u->stream>>>(u->out_train, d_target, u->dout, u->partial, nx, ny, nz, nb);
  else
    k_mse<<<mb, 256, 0, u->stream>>>(u->out_train, d_target, u->dout, u->partial, n);
  std::vector<float> lp(mb);
  HPCCG_CUDA(cudaMemcpyAsync(lp.data(), u->partial, sizeof(float) * mb, cudaMemcpyDeviceToHost, u->stream));
  HPCCG_CUDA(cudaStreamSynchronize(u->stream));
  double l = 0.0;
  for (float v : lp) l += v;
  if (loss) *loss = (float)(l / (double)n);
  if ((rc = backward(u, d_in))) return rc;
  if (grad_host) {
    HPCCG_CUDA(cudaMemcpyAsync(grad_host, u->grads, sizeof(float) * u->nparams, cudaMemcpyDeviceToHost, u->stream));
  }
  return check_err(u);
}

extern "C" int hpccg_unet_set_loss(hpccg_unet *u, int32_t kind) {
  if (!u || kind < 0 || kind > 1) return HPCCG_ERR_INVALID_ARG;
  u->loss_kind = kind;
  return HPCCG_OK;
}

extern "C" int hpccg_unet_adam_step(hpccg_unet *u, float lr, float beta1, float beta2, float eps) {
  if (!u || !(lr >= 0.f)) return HPCCG_ERR_INVALID_ARG;
  u->adam_t += 1;
  const float c1 = 1.f - powf(beta1, (float)u->adam_t), c2 = 1.f - powf(beta2, (float)u->adam_t);
  k_adam<<<grid1d(u, u->nparams), 256, 0, u->stream>>>(u->params, u->grads, u->adam_m, u->adam_v, u->nparams, lr,
                                                        beta1, beta2, eps, c1, c2);
  int rc = repack(u);
  if (rc) return rc;
  HPCCG_CUDA(cudaStreamSynchronize(u->stream));
  return HPCCG_OK;
}

extern "C" int hpccg_unet_time_forward(hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz, int32_t reps,
                                       const float *d_in, float *d_out, float *ms) {
  if (!u || reps < 1 || !ms || !d_in || !d_out) return HPCCG_ERR_INVALID_ARG;
  int rc = ensure_shape(u, nx, ny, nz, 1, false);
  if (rc) return rc;
  if ((rc = forward(u, d_in, d_out, false))) return rc;
  HPCCG_CUDA(cudaEventRecord(u->ev0, u->stream));
  for (int i = 0; i < reps; ++i)
    if ((rc = forward(u, d_in, d_out, false))) return rc;
  HPCCG_CUDA(cudaEventRecord(u->ev1, u->stream));
  HPCCG_CUDA(cudaEventSynchronize(u->ev1));
  float t = 0.f;
  HPCCG_CUDA(cudaEventElapsedTime(&t, u->ev0, u->ev1));
  *ms = t / (float)reps;
  return check_err(u);
}

// One 16-output conv layer on its own, for tests: inputs channels-last BF16
// (nin groups of 16), weights FP32 [27][16*nin][16], epilogue as ConvEpi;
// path 0 = tcgen05, 1 = CUDA cores.
extern "C" int hpccg_unet_conv3_layer(int32_t nx, int32_t ny, int32_t nz, int32_t nb, int32_t nin, const void *d_in0,
                                      const void *d_in1, const float *d_w, const float *d_bias, const float *d_proj,
                                      int32_t epi, int32_t path, void *d_out) {
  if (nin < 0 || nin > 2 || !d_in0 || (nin == 2 && !d_in1) || !d_w || !d_out || epi < 0 || epi > 3)
    return HPCCG_ERR_INVALID_ARG;
  if (nin == 0) {  // the 1-channel input layer: FP32 input [nb][nz][ny][nx], W [27][16]
    if ((epi != kEpiBiasRelu && epi != kEpiBias) || !d_bias || (path != 0 && path != 1)) return HPCCG_ERR_INVALID_ARG;
    int dev = 0, sms = 0;
    HPCCG_CUDA(cudaGetDevice(&dev));
    HPCCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const float *in = static_cast<const float *>(d_in0);
    __nv_bfloat16 *o = static_cast<__nv_bfloat16 *>(d_out);
    const int relu = epi == kEpiBiasRelu;
    int *d_err = nullptr;
    HPCCG_CUDA(cudaMalloc(&d_err, sizeof(int)));
    HPCCG_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    int rc = HPCCG_OK;
    const int64_t nvox = (int64_t)nx * ny * nz * nb;
    if (path == 0) {
      rc = launch_conv3_in1_tc(in, d_w, d_bias, o, nx, ny, nz, nb, relu, d_err, sms, 0);
    } else if (nx % 4 == 0) {
      k_conv3_in1x4<<<(int)std::min<int64_t>((nvox / 4 + 255) / 256, (int64_t)sms * 16), 256>>>(in, d_w, d_bias, o,
                                                                                              nx, ny, nz, nb, relu);
    } else {
      k_conv3_in1<<<(int)std::min<int64_t>((nvox + 255) / 256, (int64_t)sms * 16), 256>>>(in, d_w, d_bias, o, nx,
                                                                                        ny, nz, nb, relu);
    }
    if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = set_cuda_error(cudaGetLastError(), "input layer", __FILE__, __LINE__);
    int err = 0;
    cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_err);
    if (!rc && err) rc = HPCCG_ERR_TIMEOUT;
    return rc;
  }
  if ((epi != kEpiRawF32 && !d_bias) || (epi == kEpiProject && !d_proj)) return HPCCG_ERR_INVALID_ARG;
  int dev = 0, sms = 0;
  HPCCG_CUDA(cudaGetDevice(&dev));
  HPCCG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int *d_err = nullptr;
  HPCCG_CUDA(cudaMalloc(&d_err, sizeof(int)));
  HPCCG_CUDA(cudaMemset(d_err, 0, sizeof(int)));
  int rc = HPCCG_OK;
  if (path == 0 || path == 2) {
    ConvGeom g;
    if (!conv_geom(nx, ny, nz, nb, &g)) {
      cudaFree(d_err);
      return HPCCG_ERR_UNSUPPORTED;
    }
    __nv_bfloat16 *packed = nullptr;
    HPCCG_CUDA(cudaMalloc(&packed, sizeof(__nv_bfloat16) * nin * 27 * 256));
    k_pack_fwd<<<32, 256>>>(d_w, 16 * nin, nin, packed);
    ConvArgs a;
    a.g = g;
    a.in0 = static_cast<const __nv_bfloat16 *>(d_in0);
    a.in1 = static_cast<const __nv_bfloat16 *>(d_in1);
    a.wpack = packed;
    a.bias = d_bias;
    a.proj = d_proj;
    a.out = d_out;
    a.err = d_err;
    rc = launch_conv3_tc(nin, epi, a, sms, 0, path == 2);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = set_cuda_error(cudaGetLastError(), "conv3 tc", __FILE__, __LINE__);
    cudaFree(packed);
  } else {
    CcConvArgs a;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.nb = nb;
    a.nin = nin;
    a.cin = 16 * nin;
    a.in0 = static_cast<const __nv_bfloat16 *>(d_in0);
    a.in1 = static_cast<const __nv_bfloat16 *>(d_in1);
    a.in_f32 = nullptr;
    a.W = d_w;
    a.bias = d_bias;
    a.proj = d_proj;
    a.epi = epi;
    a.out = d_out;
    k_conv3_cc<<<sms * 8, 256>>>(a);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = set_cuda_error(cudaGetLastError(), "conv3 cc", __FILE__, __LINE__);
  }
  int err = 0;
  cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d_err);
  if (!rc && err) rc = HPCCG_ERR_TIMEOUT;
  return rc;
}

// Forward pass of one grid on a caller's stream (used inside solvers); no
// host synchronisation.
extern "C" int hpccg_unet_forward_on(hpccg_unet *u, int32_t nx, int32_t ny, int32_t nz, const float *d_in,
                                     float *d_out, cudaStream_t stream) {
  if (!u || !d_in || !d_out) return HPCCG_ERR_INVALID_ARG;
  int rc = ensure_shape(u, nx, ny, nz, 1, false);
  if (rc) return rc;
  cudaStream_t keep = u->stream;
  u->stream = stream;
  rc = forward(u, d_in, d_out, false);
  u->stream = keep;
  return rc;
}
