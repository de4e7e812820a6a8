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
