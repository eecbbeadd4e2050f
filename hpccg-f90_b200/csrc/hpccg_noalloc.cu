// hpccg_noalloc.cu -- a dot product that allocates nothing on the device.
//
// Some callers cannot let a library call cudaMalloc: hosts whose memory
// manager owns every byte of device memory (a pre-sized pool or a caching
// allocator that the rest of the process must go through), and code that may
// not allocate once its set-up phase is over, because cudaMalloc can
// synchronise the device and can fail on a fragmented heap.  Such callers
// cannot create an hpccg_ctx (it allocates its vectors and scratch), so this
// file offers hpccg_gpu_ddot_noalloc: the caller passes the two input arrays
// and receives the result, and the partial sums live in a fixed array that is
// part of the library image itself.
//
// The scratch array holds one partial sum per chunk of kChunk elements, so
// n is limited to kMaxPartials * kChunk = 134,217,728 elements; larger n is
// rejected with HPCCG_ERR_TOO_LARGE.  Every GPU that loads the library keeps
// this 512 KiB array (plus a few words) for the life of the process.
#include "hpccg_internal.cuh"

namespace {

constexpr int kNaBlock = 256;
constexpr int kNaPerThread = 8;
constexpr int64_t kChunk = (int64_t)kNaBlock * kNaPerThread;  // elements per partial sum
constexpr int kMaxPartials = 65536;
constexpr int64_t kMaxN = kChunk * kMaxPartials;  // 134,217,728
// Layout: [0, kMaxPartials) partial sums, [kMaxPartials] the result, and the
// arrival counter in the bits of [kMaxPartials + 1].
constexpr int kResult = kMaxPartials;
constexpr int kCounter = kMaxPartials + 1;
constexpr int kScratchWords = kMaxPartials + 32;

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[kScratchWords];

namespace {

// Block b sums elements [b*kChunk, (b+1)*kChunk) (strided by the block size, so
// loads are coalesced), writes its partial, and the last block to arrive adds
// the partials in index order: the result does not depend on scheduling.
__global__ void __launch_bounds__(kNaBlock) k_ddot_noalloc(int64_t n, const double *__restrict__ x,
                                                          const double *__restrict__ y, double *scratch) {
  __shared__ double smem[32];
  __shared__ bool s_last;
  const int64_t base = (int64_t)blockIdx.x * kChunk;
  double part = 0.0;
#pragma unroll
  for (int j = 0; j < kNaPerThread; ++j) {
    const int64_t i = base + (int64_t)j * kNaBlock + threadIdx.x;
    if (i < n) part = __dadd_rn(part, __dmul_rn(__ldg(x + i), __ldg(y + i)));
  }
  const double tot = hpccg::block_sum<kNaBlock>(part, smem);
  unsigned *counter = reinterpret_cast<unsigned *>(scratch + kCounter);
  if (threadIdx.x == 0) {
    scratch[blockIdx.x] = tot;
    __threadfence();
    s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kNaBlock)
    v = __dadd_rn(v, ((volatile double *)scratch)[i]);
  v = hpccg::block_sum<kNaBlock>(v, smem);
  if (threadIdx.x == 0) {
    scratch[kResult] = v;
    *counter = 0u;
  }
}

// Device address of the scratch array on the current device.  The name
// g_noalloc_scratch in host code is only a host-side stand-in, not a device
// address, so every call asks the runtime for the address on the device that
// is current now.  The lookup is cheap next to the call's synchronisation, and
// unlike an address cached per device index it stays right after the device's
// context is re-created (cudaDeviceReset re-loads the library's module, and the
// array may then sit elsewhere).
int scratch_for_current_device(double **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return hpccg::set_cuda_error(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
  *out = static_cast<double *>(p);
  return HPCCG_OK;
}

}  // namespace

extern "C" int hpccg_gpu_ddot_noalloc(int32_t n, const double *d_x, const double *d_y, double *result,
                                      void *stream) {
  if (n < 0 || !result || (n > 0 && (!d_x || !d_y))) return HPCCG_ERR_INVALID_ARG;
  if ((int64_t)n > kMaxN) return HPCCG_ERR_TOO_LARGE;
  if (n == 0) {
    *result = 0.0;
    return HPCCG_OK;
  }
  double *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The counter must start at zero; partial slots are always written before read.
  HPCCG_CUDA(cudaMemsetAsync(scratch + kCounter, 0, sizeof(double), s));
  const int blocks = (int)((n + kChunk - 1) / kChunk);
  k_ddot_noalloc<<<blocks, kNaBlock, 0, s>>>(n, d_x, d_y, scratch);
  HPCCG_CUDA(cudaGetLastError());
  HPCCG_CUDA(cudaMemcpyAsync(result, scratch + kResult, sizeof(double), cudaMemcpyDeviceToHost, s));
  HPCCG_CUDA(cudaStreamSynchronize(s));
  return HPCCG_OK;
}
