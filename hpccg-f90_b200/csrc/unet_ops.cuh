// unet_ops.cuh -- declarations of the CUDA-core U-Net kernels (unet_ops.cu).
#pragma once
#include "unet_conv.cuh"

namespace hpccg {

struct CcConvArgs {
  int nx, ny, nz, nb;
  int nin, cin;                      // 16-channel input groups and total input channels
  const __nv_bfloat16 *in0, *in1;    // row-planar BF16 inputs
  const float *in_f32;               // or a 1-channel FP32 input (cin = 1)
  const float *W;                    // FP32 [27][cin][16]
  const float *bias;                 // [16] or null
  const float *proj;                 // [17] for kEpiProject
  int epi;
  void *out;
};

struct DwArgs {
  int nx, ny, nz, nb, cin;
  const __nv_bfloat16 *x0, *x1;      // forward inputs (channels 0-15, 16-31)
  const float *x_f32;                // or the 1-channel FP32 input
  const __nv_bfloat16 *dy;           // gradient w.r.t. the pre-activation output
  float *partial;                    // [gridDim.x][27*cin + 1][16]
};

__global__ void k_pack_fwd(const float *W, int cin, int nin, __nv_bfloat16 *packed);
__global__ void k_pack_bwd(const float *W, int cin, int g, __nv_bfloat16 *packed);
__global__ void k_flip_fp32(const float *W, int cin, int g, float *Wf);
__global__ void k_conv3_cc(CcConvArgs a);
__global__ void k_conv3_in1(const float *in, const float *W, const float *bias, __nv_bfloat16 *out, int nx, int ny,
                            int nz, int nb, int relu);
__global__ void k_conv3_in1x4(const float *in, const float *W, const float *bias, __nv_bfloat16 *out, int nx, int ny,
                              int nz, int nb, int relu);  // nx a multiple of 4
__global__ void k_pool(const __nv_bfloat16 *in, __nv_bfloat16 *out, int nx, int ny, int nz, int nb);
__global__ void k_upsample(const __nv_bfloat16 *in, __nv_bfloat16 *out, int nx, int ny, int nz, int nb);
__global__ void k_pool_bwd(const float *dc, float *df, int nx, int ny, int nz, int nb);
__global__ void k_up_bwd(const float *df, float *dc, int nx, int ny, int nz, int nb);
__global__ void k_relu_mask(const float *d, const __nv_bfloat16 *act, __nv_bfloat16 *out, int64_t n);
__global__ void k_add_f32(const float *src, float *dst, int64_t n);
__global__ void k_dW(DwArgs a);
__global__ void k_reduce_partials(const float *partial, int nblocks, int n, float *grad, int accumulate);
__global__ void k_proj_fwd(const __nv_bfloat16 *act, const float *proj, float *out, int64_t nvox, int nx);
__global__ void k_proj_bwd(const __nv_bfloat16 *act, const float *proj, const float *dout, __nv_bfloat16 *dact,
                           float *partial, int64_t nvox, int nx);
__global__ void k_mse(const float *out, const float *tgt, float *dout, float *partial, int64_t n);
__global__ void k_energy(const float *out, const float *tgt, float *dout, float *partial, int nx, int ny, int nz,
                         int nb);
__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2);

}  // namespace hpccg
