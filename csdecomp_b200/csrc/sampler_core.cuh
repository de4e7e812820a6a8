// sampler_core.cuh -- one hit-and-run chain, shared by the sampler and the
// batched EI-ZO kernels.
#pragma once
#include <cfloat>

#include "csd_rng.cuh"

namespace csd {

// One hit-and-run chain (cuda_hit_and_run_sampling.cu:57-118): returns false
// if a line search found an empty theta interval. x holds the start on entry.
template <int MAXD>
__device__ __forceinline__ bool run_chain(const float* __restrict__ Ap, const float* __restrict__ bp, int F, int dim,
                                          int mixing, uint32_t k0, uint32_t k1, uint32_t chain, uint32_t stream,
                                          float* x) {
  float dir[MAXD];
#pragma unroll
  for (int k = 0; k < MAXD; ++k) dir[k] = 0.f;
  for (int step = 0; step < mixing; ++step) {
    float ut;
    step_draws<MAXD>(k0, k1, chain, stream, (uint32_t)step, dim, dir, &ut);
    float tmax = FLT_MAX, tmin = -FLT_MAX;
    for (int f = 0; f < F; ++f) {
      const float* a = Ap + (int64_t)f * dim;
      float ax = __fmul_rn(a[0], x[0]);
      float ad = __fmul_rn(a[0], dir[0]);
#pragma unroll
      for (int k = 1; k < MAXD; ++k) {
        if (k < dim) {
          float ak = a[k];
          ax = __fmaf_rn(ak, x[k], ax);
          ad = __fmaf_rn(ak, dir[k], ad);
        }
      }
      float lb = __fsub_rn(bp[f], ax);
      if (ad < 0.0f)
        tmin = fmaxf(tmin, __fdiv_rn(lb, ad));
      else if (ad > 0.0f)
        tmax = fminf(tmax, __fdiv_rn(lb, ad));
    }
    if (isinf(tmax) || isinf(tmin) || tmax < tmin) return false;
    double th = __dadd_rn(__dmul_rn((double)ut, __dsub_rn(__dmul_rn(0.999999, (double)tmax), (double)tmin)),
                          (double)tmin);
    float theta = __double2float_rn(th);
#pragma unroll
    for (int k = 0; k < MAXD; ++k)
      if (k < dim) x[k] = __fmaf_rn(theta, dir[k], x[k]);
  }
  return true;
}

}  // namespace csd
