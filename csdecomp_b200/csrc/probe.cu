// probe.cu -- FP32 FMA throughput probe: the denominator of the collision
// kernels' FP32 roofline (the driver-measured peaks cover HBM and BF16 only).
#include "csd_internal.h"

namespace csd {

// 8 independent FMA chains per thread; the result is written so the chains stay live.
__global__ void __launch_bounds__(256) fma_probe_kernel(int64_t iters, float* out) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  const float m = 0.9999999f, c = 1e-7f;
  for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

}  // namespace csd

extern "C" csd_status_t csd_fp32_fma_probe(int64_t iters, double* flops, double* seconds) {
  using namespace csd;
  CSD_CHECK(flops && seconds && iters > 0, CSD_ERR_INVALID, "null argument");
  const int sms = device_sm_count();
  const int blocks = sms * 8, threads = 256;
  float* out = nullptr;
  CSD_CUDA_TRY(cudaMalloc(&out, sizeof(float) * blocks * threads));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_probe_kernel<<<blocks, threads>>>(iters / 8 + 1, out);  // warm-up
  cudaEventRecord(e0);
  fma_probe_kernel<<<blocks, threads>>>(iters, out);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) {
    set_error(cudaGetErrorString(err));
    return CSD_ERR_CUDA;
  }
  *seconds = ms * 1e-3;
  *flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  return CSD_OK;
}
