// sampler.cu -- hit-and-run sampling in H-polytopes.
//
// Reference: uniformSampleInHPolyhedronKernel, one thread per sample chain,
// cuda_hit_and_run_sampling.cu:18-119: a Gaussian direction per mixing step,
// slack b - A x and A dir per face, theta interval from the sign of (A dir)_i,
// theta = u * (0.999999 * theta_max - theta_min) + theta_min (:106-107).
// Same chain structure here; the face loop reads A and b with warp-uniform
// addresses (every thread of a polytope walks the same face at the same time,
// so each load is one broadcast transaction), keeps the chain state in
// registers (the reference keeps two float[4000] arrays per thread in local
// memory) and draws from the counter-based stream of csd_rng.cuh.
#include <algorithm>
#include <cfloat>

#include "csd_internal.h"
#include "csd_rng.cuh"
#include "sampler_core.cuh"

namespace csd {

template <int MAXD>
__global__ void __launch_bounds__(128) hit_and_run_kernel(const float* __restrict__ A, const float* __restrict__ b,
                                                          const int32_t* __restrict__ face_off,
                                                          const int* __restrict__ num_faces_dev, int num_poly,
                                                          int dim, const float* __restrict__ starts, int S,
                                                          int mixing, uint32_t k0, uint32_t k1,
                                                          uint32_t stream_base, int fail_keep,
                                                          float* __restrict__ out, int* num_failed) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)num_poly * S) return;
  const int poly = (int)(i / S);
  const int s = (int)(i % S);
  const int f0 = face_off ? face_off[poly] : 0;
  const int F = face_off ? face_off[poly + 1] - f0 : *num_faces_dev;
  float x[MAXD];
#pragma unroll
  for (int k = 0; k < MAXD; ++k) x[k] = k < dim ? starts[(int64_t)poly * dim + k] : 0.f;
  const bool ok = run_chain<MAXD>(A + (int64_t)f0 * dim, b + f0, F, dim, mixing, k0, k1, (uint32_t)s,
                                  stream_base + (uint32_t)poly, x);
  if (!ok && num_failed) atomicAdd(num_failed, 1);
  // a chain whose line search fails writes NaN, or (fail_keep) its start point
  float* dst = out + i * dim;
#pragma unroll
  for (int k = 0; k < MAXD; ++k)
    if (k < dim) dst[k] = ok ? x[k] : fail_keep ? starts[(int64_t)poly * dim + k] : __int_as_float(0x7fc00000);
}

// Group-per-chain sampler over one polytope given transposed (At[k * ldt +
// f]); the face count is read on the device. Used by the inflator, whose
// region grows to hundreds of faces: the polytope is staged in shared memory
// once per block (as face rows while they fit, else as transposed columns)
// and the lanes of a group share the face loop.
__global__ void __launch_bounds__(256) hit_and_run_group_kernel(const float* __restrict__ At, int ldt,
                                                                const float* __restrict__ b,
                                                                const int* __restrict__ num_faces_dev, int dim,
                                                                const float* __restrict__ start, int S, int mixing,
                                                                uint32_t k0, uint32_t k1, uint32_t stream,
                                                                float* __restrict__ out) {
  extern __shared__ __align__(16) float smf[];  // the face loop reads float2/float4 vectors
  const int F = *num_faces_dev;
  const int G = group_width(S, (int64_t)gridDim.x * (blockDim.x >> 5));
  const int per = (S + gridDim.x - 1) / gridDim.x;
  const int first = blockIdx.x * per, last = min(S, first + per);
  if (first >= last) return;
  constexpr int rows8 = (int)(kStageBytes / (kRowStride<8> * sizeof(float)));
  constexpr int rows16 = (int)(kStageBytes / (kRowStride<16> * sizeof(float)));
  if (dim <= 8) {
    if (F <= rows8) {
      stage_rows<8>(At, ldt, b, F, dim, smf);
      __syncthreads();
      sample_range<8, 1, kLayRows>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out, G, smf, true);
      return;
    }
    const bool staged = F <= kStageFaces8;
    if (staged) stage_polytope<8, kStageFaces8>(At, ldt, b, F, dim, smf);
    __syncthreads();
    sample_range<8, 1>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out, G, smf, staged);
  } else {
    if (F <= rows16) {
      stage_rows<16>(At, ldt, b, F, dim, smf);
      __syncthreads();
      sample_range<16, 1, kLayRows>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out, G, smf, true);
      return;
    }
    const bool staged = F <= kStageFaces16;
    if (staged) stage_polytope<16, kStageFaces16>(At, ldt, b, F, dim, smf);
    __syncthreads();
    sample_range<16, 1>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out, G, smf, staged);
  }
}

csd_status_t launch_hit_and_run_warp(const float* At, int ldt, const float* b, const int* num_faces_dev, int dim,
                                     const float* start, int S, int mixing, uint64_t seed, uint32_t stream,
                                     int fail_keep, float* out, cudaStream_t st) {
  if (S <= 0) return CSD_OK;
  CSD_CHECK(dim >= 1 && dim <= kMaxDim, CSD_ERR_DIMENSION, "dimension must be in [1, 16]");
  CSD_CHECK(fail_keep, CSD_ERR_INVALID, "the group sampler keeps the start point of failed chains");
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr_set[dev]) {
    CSD_CUDA_TRY(cudaFuncSetAttribute(hit_and_run_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kStageBytes));
    if (dev < 64) attr_set[dev] = true;
  }
  const int sms = device_sm_count();
  const int blocks = (int)std::min<int64_t>(((int64_t)S + 7) / 8, (int64_t)sms * 2);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  hit_and_run_group_kernel<<<blocks, 256, kStageBytes, st>>>(At, ldt, b, num_faces_dev, dim, start, S, mixing, k0,
                                                              k1, stream, out);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

// Transposes F rows of A (row-major, d columns) into At (At[k * ldt + f]).
__global__ void transpose_faces_kernel(const float* __restrict__ A, int F, int d, float* __restrict__ At, int ldt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F * d; i += gridDim.x * blockDim.x)
    At[(int64_t)(i % d) * ldt + i / d] = A[i];
}

csd_status_t launch_transpose_faces(const float* A, int F, int d, float* At, int ldt, cudaStream_t st) {
  if (F <= 0) return CSD_OK;
  const int blocks = std::min((F * d + 255) / 256, 1024);
  transpose_faces_kernel<<<blocks, 256, 0, st>>>(A, F, d, At, ldt);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_hit_and_run(const float* A, const float* b, const int32_t* face_off, int num_poly, int dim,
                                const float* starts, int S, int mixing, uint64_t seed, uint32_t stream_base,
                                int fail_keep, float* out, int* num_failed, const int* num_faces_dev,
                                cudaStream_t st) {
  const int64_t total = (int64_t)num_poly * S;
  if (total <= 0) return CSD_OK;
  CSD_CHECK(dim >= 1 && dim <= kMaxDim, CSD_ERR_DIMENSION, "dimension must be in [1, 16]");
  const int threads = 128;
  const int64_t blocks = (total + threads - 1) / threads;
  CSD_CHECK(blocks < (1ll << 31), CSD_ERR_CAPACITY, "too many samples");
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#define CSD_HR(MD)                                                                                         \
  hit_and_run_kernel<MD><<<(unsigned)blocks, threads, 0, st>>>(A, b, face_off, num_faces_dev, num_poly, dim, \
                                                               starts, S, mixing, k0, k1, stream_base,     \
                                                               fail_keep, out, num_failed)
  if (dim <= 2)
    CSD_HR(2);
  else if (dim <= 4)
    CSD_HR(4);
  else if (dim <= 8)
    CSD_HR(8);
  else
    CSD_HR(16);
#undef CSD_HR
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

}  // namespace csd
