// csd_rng.cuh -- the sampler's random stream.
//
// The reference seeds cuRAND XORWOW per thread (cuda_hit_and_run_sampling.cu:26)
// and draws curand_normal/curand_uniform. This build specifies its own
// counter-based stream so that every draw is a pure function of
// (seed, chain, stream, step) and reproducible on the CPU:
//   * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//     easy as 1, 2, 3", SC'11); key = (seed lo, seed hi),
//     counter = (step, chain, stream, block);
//   * uniform in (0,1]: ((x >> 8) + 1) * 2^-24, angle fraction in [0,1): (x >> 8) * 2^-24;
//   * Gaussian pairs by Box-Muller with this file's ln() (atanh series) and
//     sin/cos of 2*pi*v (Taylor series), every operation an explicitly
//     rounded IEEE-754 single-precision op (no contraction), so results are
//     bit-identical to a C++ implementation of the same steps.
#pragma once
#include <cstdint>

namespace csd {

__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                              uint32_t k1, uint32_t* out) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    // one 32 x 32 -> 64-bit multiply per word (a single wide integer multiply-add)
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

__device__ __forceinline__ float u01_open0(uint32_t x) {
  return __fmul_rn((float)((x >> 8) + 1u), 5.9604644775390625e-08f);
}
__device__ __forceinline__ float u01_open1(uint32_t x) { return __fmul_rn((float)(x >> 8), 5.9604644775390625e-08f); }

// ln(u), u in (0,1]: u = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
// s = (m-1)/(m+1); ln 2 = 0.693145751953125 + 1.4286067653301870e-06 (head exact in products with e).
__device__ __forceinline__ float log_unit(float u) {
  uint32_t bits = __float_as_uint(u);
  int e = (int)(bits >> 23) - 127;
  float m = __uint_as_float((bits & 0x007fffffu) | 0x3f800000u);
  const bool hi = m > 1.41421353816986083984375f;  // selects, not a branch (lanes draw different u)
  m = hi ? __fmul_rn(m, 0.5f) : m;
  e += hi ? 1 : 0;
  float s = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
  float s2 = __fmul_rn(s, s);
  float p = __fmaf_rn(s2, 0.0909090936183929443359375f, 0.111111111938953399658203125f);
  p = __fmaf_rn(s2, p, 0.142857149243354797363281250f);
  p = __fmaf_rn(s2, p, 0.20000000298023223876953125f);
  p = __fmaf_rn(s2, p, 0.3333333432674407958984375f);
  p = __fmaf_rn(s2, p, 1.0f);
  float t = __fmul_rn(s, p);
  float lnm = __fadd_rn(t, t);
  float fe = (float)e;
  float lo = __fmaf_rn(fe, 1.428606765330187045037746429443359375e-06f, lnm);
  return __fmaf_rn(fe, 0.693145751953125f, lo);
}

// (sin, cos) of 2*pi*v, v in [0,1): quadrant from 4v, x = f*pi/2, Taylor
// series through x^13 (sin) and x^14 (cos), Horner in x^2.
__device__ __forceinline__ void sincos_2pi(float v, float* sn, float* cs) {
  float w = __fmul_rn(v, 4.0f);
  int qd = (int)w;
  float f = __fsub_rn(w, (float)qd);
  float x = __fmul_rn(f, 1.57079637050628662109375f);
  float x2 = __fmul_rn(x, x);
  float ps = __fmaf_rn(x2, 1.6059043836821614e-10f, -2.5052108385441720e-08f);
  ps = __fmaf_rn(x2, ps, 2.7557319223985893e-06f);
  ps = __fmaf_rn(x2, ps, -1.9841269841269841e-04f);
  ps = __fmaf_rn(x2, ps, 8.3333333333333333e-03f);
  ps = __fmaf_rn(x2, ps, -1.6666666666666667e-01f);
  ps = __fmaf_rn(x2, ps, 1.0f);
  float s = __fmul_rn(x, ps);
  float pc = __fmaf_rn(x2, -1.1470745597729725e-11f, 2.0876756987868099e-09f);
  pc = __fmaf_rn(x2, pc, -2.7557319223985891e-07f);
  pc = __fmaf_rn(x2, pc, 2.4801587301587302e-05f);
  pc = __fmaf_rn(x2, pc, -1.3888888888888889e-03f);
  pc = __fmaf_rn(x2, pc, 4.1666666666666667e-02f);
  pc = __fmaf_rn(x2, pc, -0.5f);
  float c = __fmaf_rn(x2, pc, 1.0f);
  // quadrant qd: (sin, cos) = (s, c), (c, -s), (-s, -c), (-c, s), by selects
  const float ss = (qd & 1) ? c : s, cc = (qd & 1) ? s : c;
  *sn = (qd & 2) ? -ss : ss;
  *cs = ((qd + 1) & 2) ? -cc : cc;
}

// Direction (dim Gaussians) and the theta uniform of one mixing step.
// Gaussian pair g uses words 2g (radius) and 2g+1 (angle); the theta uniform
// is word 2*ceil(dim/2). Words 4k..4k+3 come from Philox block k.
template <int MAXD>
__device__ __forceinline__ void step_draws(uint32_t k0, uint32_t k1, uint32_t chain, uint32_t stream, uint32_t step,
                                           int dim, float* dir, float* u_theta) {
  const int npairs = (dim + 1) >> 1;
  uint32_t w[4];
  int have_block = -1;
#pragma unroll
  for (int g = 0; g < (MAXD + 1) / 2; ++g) {
    if (g < npairs) {
      int blk = (2 * g) >> 2;
      if (blk != have_block) {
        philox4x32_10(step, chain, stream, (uint32_t)blk, k0, k1, w);
        have_block = blk;
      }
      float u = u01_open0(w[(2 * g) & 3]);
      float v = u01_open1(w[(2 * g + 1) & 3]);
      float rad = __fsqrt_rn(__fmul_rn(-2.0f, log_unit(u)));
      float sn, cs;
      sincos_2pi(v, &sn, &cs);
      dir[2 * g] = __fmul_rn(rad, cs);
      if (2 * g + 1 < MAXD) dir[2 * g + 1] = __fmul_rn(rad, sn);
    }
  }
  int tw = 2 * npairs;
  int blk = tw >> 2;
  if (blk != have_block) philox4x32_10(step, chain, stream, (uint32_t)blk, k0, k1, w);
  *u_theta = u01_open0(w[tw & 3]);
}

}  // namespace csd
