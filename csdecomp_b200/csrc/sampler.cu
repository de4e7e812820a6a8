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
#include <atomic>
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

// EI-ZO sampler over one region (the single inflation and the
// allocation-free inflation), whose face count is read on the device: the
// region's face-pair rows are staged in shared memory once per block when
// they fit (else the chains read them from global memory, through L1), and
// the block's chains run with G lanes each (sampler_core.cuh; G from the
// chain count, widened so that a lane holds at most kRegionKP face pairs).
constexpr int kRegionKP = 8;
constexpr size_t kRegionStageBytes = 104 * 1024;  // two blocks per SM
static_assert(kMaxRegionFaces <= 2 * 256 * kRegionKP, "the widest group samples the largest region");

__global__ void __launch_bounds__(256, 2) sample_region_kernel(const float* __restrict__ rows,
                                                              const int* __restrict__ num_faces_dev, int dim,
                                                              const float* __restrict__ start, int S, int mixing,
                                                              uint32_t k0, uint32_t k1, uint32_t stream,
                                                              float* __restrict__ out) {
  extern __shared__ __align__(16) float smf[];  // the face loop reads 16-byte vectors
  __shared__ GroupScratch gsa[kMaxWideGroups];
  const int F = *num_faces_dev;
  const int P = (F + 1) >> 1, rs = pair_stride(dim);
  const int G = pair_group_width(group_width(S, (int64_t)gridDim.x * (blockDim.x >> 5)), P, kRegionKP);
  const int per = (S + gridDim.x - 1) / gridDim.x;
  const int first = blockIdx.x * per, last = min(S, first + per);
  if (first >= last || G == 0) return;  // uniform across the block (the host bounds F)
  const bool fits = (size_t)P * rs * sizeof(float) <= kRegionStageBytes;
  if (fits) {
    stage_pairs(rows, P, rs, smf);
    __syncthreads();
  }
  // separate calls for staged and global rows (shared-memory loads in the staged face loop)
  if (fits) {
    if (dim <= 8)
      sample_region<8, kRegionKP>(G, smf, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
    else
      sample_region<16, kRegionKP>(G, smf, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
  } else {
    if (dim <= 8)
      sample_region<8, kRegionKP>(G, rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
    else
      sample_region<16, kRegionKP>(G, rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
  }
}

csd_status_t launch_sample_region(const float* rows, const int* num_faces_dev, int dim, const float* start, int S,
                                  int mixing, uint64_t seed, uint32_t stream, float* out, cudaStream_t st) {
  if (S <= 0) return CSD_OK;
  CSD_CHECK(dim >= 1 && dim <= kMaxDim, CSD_ERR_DIMENSION, "dimension must be in [1, 16]");
  static std::atomic<bool> attr_set[64] = {};  // per device: limit raised (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr_set[dev]) {
    CSD_CUDA_TRY(raise_smem_limit(sample_region_kernel, (int)kRegionStageBytes));
    if (dev < 64) attr_set[dev] = true;
  }
  const int sms = device_sm_count();
  const int blocks = (int)std::min<int64_t>(((int64_t)S + 7) / 8, (int64_t)sms * 2);
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  sample_region_kernel<<<blocks, 256, kRegionStageBytes, st>>>(rows, num_faces_dev, dim, start, S, mixing, k0, k1,
                                                                stream, out);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

__global__ void put_faces_kernel(const float* __restrict__ A, const float* __restrict__ b, int F, int dim,
                                 const float* __restrict__ x0, float* __restrict__ rows) {
  put_faces(A, b, F, dim, x0, rows, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

csd_status_t launch_put_faces(const float* A, const float* b, int F, int dim, const float* x0, float* rows,
                              cudaStream_t st) {
  if (F <= 0) return CSD_OK;
  const int pairs = (F + 1) / 2;
  put_faces_kernel<<<(pairs + 127) / 128, 128, 0, st>>>(A, b, F, dim, x0, rows);
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
