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

// ---- packed FP32 pairs (sm_100 f32x2): each half is an IEEE round-to-nearest
// operation, so a packed result is bit for bit the two scalar results.
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float* lo, float* hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(*lo), "=f"(*hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// ---------------------------------------------------------------------------
// EI-ZO sampling: hit-and-run with carried slacks over face pairs.
//
// Every chain of an EI-ZO iteration starts at the segment's start point x0,
// so the slack b_f - a_f . x0 of a face at the start of a chain is common to
// all chains. It is computed once, when the face is written (put_face), in the
// serial chain's order (product of coordinate 0, fused multiply-adds in
// coordinate order, then b minus that). A chain carries its slacks: after a
// step of length theta along dir it updates s_f = fma(-theta, a_f . dir, s_f),
// so a mixing step costs one dim-long dot product per face instead of two
// (the reference recomputes b - A x every step,
// csdecomp/src/planning/cuda_hit_and_run_sampling.cu:83-104). The theta
// bounds, the theta draw (0.999999 scales theta_max only, :106-107) and the
// position update are the serial chain's.
//
// Face-pair rows: row p holds faces 2p and 2p + 1 interleaved, coordinate k of
// face 2p + h at float 2k + h (k < MAXD, zero past dim), the two start slacks
// at 2 MAXD and 2 MAXD + 1, then two unused floats: 2 MAXD + 4 floats, a
// multiple of 16 bytes. A face that does not exist yet (the partner of the
// last face of an odd count) holds a copy of that face: it bounds theta
// exactly as the face does, so it changes no bound. One 16-byte load brings two
// coordinates of both faces, and one packed FMA (fma.rn.f32x2, each half an
// IEEE round-to-nearest FMA) advances both faces' dot products.
__host__ __device__ constexpr int pair_maxd(int dim) { return dim <= 8 ? 8 : 16; }
__host__ __device__ constexpr int pair_stride(int dim) { return 2 * pair_maxd(dim) + 4; }

// Writes face f (coordinates a[0..dim), offset b) of a region whose chains
// start at x0. An even f also fills its partner half with a copy of itself.
__device__ __forceinline__ void put_face(float* __restrict__ rows, int dim, int f, const float* a, float b,
                                         const float* __restrict__ x0) {
  const int md = pair_maxd(dim), h = f & 1;
  float* r = rows + (size_t)(f >> 1) * pair_stride(dim);
  float ax = __fmul_rn(a[0], x0[0]);
  for (int k = 1; k < dim; ++k) ax = __fmaf_rn(a[k], x0[k], ax);
  for (int k = 0; k < md; ++k) r[2 * k + h] = k < dim ? a[k] : 0.f;
  r[2 * md + h] = __fsub_rn(b, ax);
  if (!h) {  // until face f + 1 is written, its half repeats face f (a face seen twice bounds nothing new)
    for (int k = 0; k < md; ++k) r[2 * k + 1] = r[2 * k];
    r[2 * md + 1] = r[2 * md];
  }
}

// Pair rows of faces [0, F) of a row-major A (F x dim) and b; thread t of
// nthreads writes whole pairs t, t + nthreads, ...
__device__ __forceinline__ void put_faces(const float* __restrict__ A, const float* __restrict__ b, int F, int dim,
                                          const float* __restrict__ x0, float* __restrict__ rows, int t,
                                          int nthreads) {
  for (int p = t; p < (F + 1) / 2; p += nthreads) {
    put_face(rows, dim, 2 * p, A + (size_t)(2 * p) * dim, b[2 * p], x0);
    if (2 * p + 1 < F) put_face(rows, dim, 2 * p + 1, A + (size_t)(2 * p + 1) * dim, b[2 * p + 1], x0);
  }
}

// theta bounds of one face (slack s, a . dir = ad): the reference's rule
// (ad < 0 raises theta_min to s / ad, ad > 0 lowers theta_max to s / ad, ad = 0
// bounds nothing), as one IEEE division and two selects, so that lanes whose
// faces point either way do not split into two division paths. For ad = 0
// (either sign) the quotient is infinite or NaN and neither select takes it;
// the rows hold no zero faces (an unpaired face is repeated), so that case,
// which takes the division's slow path, only arises when a . dir is exactly 0.
__device__ __forceinline__ void theta_bound(float s, float ad, float& tmin, float& tmax) {
  const float q = __fdiv_rn(s, ad);
  tmin = ad < 0.0f ? fmaxf(tmin, q) : tmin;
  tmax = ad > 0.0f ? fminf(tmax, q) : tmax;
}

// Steps whose draws a group computes at once (when its drawing lanes hold
// that many steps' jobs).
constexpr int kDrawSteps = 8;

// Shared scratch of a group wider than a warp (G = 64, 128, 256 lanes): the
// directions and theta uniforms of a batch of drawn steps (coordinates 0..15,
// the uniform at 16), double buffered by batch parity, and each warp's
// partial theta bounds, double buffered by step parity (a warp cannot run two
// steps, or two batches, ahead of the group's barriers).
struct GroupScratch {
  float dir[2][kDrawSteps][17];
  float red[2][8][2];
};
constexpr int kMaxWideGroups = 4;  // 256 threads / 64 lanes

__device__ __forceinline__ void group_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Lanes per chain: at least `g` (set by the chain count) and enough that
// each lane holds at most KP face pairs; 0 if even 256 lanes do not.
__host__ __device__ __forceinline__ int pair_group_width(int g, int P, int KP) {
  while (g <= 256 && (long long)g * KP < P) g <<= 1;
  return g <= 256 ? g : 0;
}

// One chain run by a group of G lanes over a region of P face pairs (staged in
// shared memory or read from global memory). Lane gl holds pairs gl + G j
// (j < KP) and their slacks and a . dir values in registers, and coordinates
// gl + G r of the position (xl). The draws are the serial chain's: step s
// reads words 0 .. 2 ceil(dim/2) of its stream (Gaussian pair j from words 2j
// and 2j + 1, the theta uniform from word 2 ceil(dim/2)), four words per
// Philox block. A drawing slot is one block: both its Box-Muller pairs (or a
// pair and the theta uniform). A step has JB = ceil(dim/2) / 2 + 1 blocks; the
// group's drawing lanes (all of a group of up to 32, the first warp of a wider
// one) draw S = min(kDrawSteps, lanes / JB) steps at once, slot q = gl holding
// block q % JB of step offset q / JB, so Gaussian pair p of offset t lies on
// lane t JB + p / 2. The direction reaches the group by shuffles (G <= 32) or
// through GroupScratch (wider groups, named barrier bar_id). The theta bounds
// are max/min reductions, which do not depend on the order, so every chain
// ends bit for bit where the oracle's serial chain ends whatever G. A chain
// whose line search fails keeps stepping without moving (the group's lanes
// stay convergent) and returns false.
template <int MAXD, int G, int KP>
__device__ __forceinline__ bool run_chain_pairs(const float* __restrict__ rows, int P, int dim, int mixing,
                                                uint32_t k0, uint32_t k1, uint32_t chain, uint32_t stream,
                                                float* xl, int gl, GroupScratch* gs, int bar_id) {
  constexpr int RS = 2 * MAXD + 4;
  constexpr int GD = G < 32 ? G : 32;    // drawing lanes
  constexpr int XL = (MAXD + G - 1) / G;  // position coordinates per lane
  static_assert(MAXD / 4 + 1 <= GD, "one step's blocks fit the drawing lanes");
  const int npairs = (dim + 1) >> 1, JB = (npairs >> 1) + 1;
  const int S = min(kDrawSteps, GD / JB);  // steps drawn at once (uniform)
  const int tq = gl / JB, bq = gl - tq * JB;  // this lane's slot: step offset, block
  // a lane past the last pair in round j holds a copy of pair P - 1 there: its work is the same
  // as that pair's owner's (so the group's lanes never diverge in the face loop) and a face seen
  // twice changes no theta bound
  uint64_t s2[KP], a2[KP];
#pragma unroll
  for (int j = 0; j < KP; ++j) {
    const int p = min(gl + G * j, P - 1);
    s2[j] = P > 0 ? *reinterpret_cast<const uint64_t*>(rows + (size_t)p * RS + 2 * MAXD) : 0ull;
    a2[j] = 0ull;  // with nth = -0 the first update leaves every slack as it is
  }
  float nth = -0.0f;
  bool ok = true;
  // this lane's block: pair 2 bq (c0a, c1a) and pair 2 bq + 1 (c0b, c1b); where a pair index
  // reaches npairs its c0 holds the theta uniform instead
  float c0a = 0.f, c1a = 0.f, c0b = 0.f, c1b = 0.f;
  int t = 0, batch = -1;  // step offset within the drawn batch, batch parity
  for (int step = 0; step < mixing; ++step) {
    if (t == 0) {
      ++batch;
      // wide groups draw in their first warp (uniform across a warp); every drawing lane
      // evaluates its slot without branching (lanes past the batch's last slot compute values
      // nobody reads), so the group's lanes stay convergent through the draws
      if (G <= 32 || gl < 32) {
        uint32_t w[4];
        philox4x32_10((uint32_t)(step + tq), chain, stream, (uint32_t)bq, k0, k1, w);
        const float ua = u01_open0(w[0]), ub = u01_open0(w[2]);
        const float rada = __fsqrt_rn(__fmul_rn(-2.0f, log_unit(ua)));
        const float radb = __fsqrt_rn(__fmul_rn(-2.0f, log_unit(ub)));
        float sna, csa, snb, csb;
        sincos_2pi(u01_open1(w[1]), &sna, &csa);
        sincos_2pi(u01_open1(w[3]), &snb, &csb);
        const bool ga = 2 * bq < npairs, gb = 2 * bq + 1 < npairs;
        c0a = ga ? __fmul_rn(rada, csa) : ua;
        c1a = __fmul_rn(rada, sna);
        c0b = gb ? __fmul_rn(radb, csb) : ub;
        c1b = __fmul_rn(radb, snb);
      }
      if constexpr (G > 32) {
        if (gl < S * JB) {  // the first warp's lanes (S JB <= 32)
          float* db = gs->dir[batch & 1][tq];
          if (2 * bq < npairs) {
            db[4 * bq] = c0a;
            db[4 * bq + 1] = c1a;
          } else {
            db[16] = c0a;
          }
          if (2 * bq + 1 < npairs) {
            db[4 * bq + 2] = c0b;
            db[4 * bq + 3] = c1b;
          } else if (2 * bq + 1 == npairs) {
            db[16] = c0b;
          }
        }
      }
    }
    const int base = t * JB;  // lane of this step's block 0
    uint64_t dd[MAXD];        // (dir_k, dir_k)
    float ut;
    if constexpr (G <= 32) {
#pragma unroll
      for (int k = 0; k < MAXD; ++k) {
        // coordinate k: pair k >> 1 = block k >> 2, half (k >> 1) & 1, cosine or sine k & 1
        const float v = ((k >> 1) & 1) ? ((k & 1) ? c1b : c0b) : ((k & 1) ? c1a : c0a);
        const float dk = __shfl_sync(0xffffffffu, v, base + (k >> 2), G);
        dd[k] = f2_pack(dk, dk);
      }
      const float utv = (npairs & 1) ? c0b : c0a;  // the theta uniform: block npairs / 2, half npairs & 1
      ut = __shfl_sync(0xffffffffu, utv, base + (npairs >> 1), G);
    } else {
      const float* db = gs->dir[batch & 1][t];
      if (t == 0) group_bar(bar_id, G);  // the batch's draws are in scratch
#pragma unroll
      for (int k = 0; k < MAXD; ++k) {
        const float dk = db[k];  // entries past dim are never used
        dd[k] = f2_pack(dk, dk);
      }
      ut = db[16];
    }
    float tmax = FLT_MAX, tmin = -FLT_MAX;
    const uint64_t nth2 = f2_pack(nth, nth);
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      if (G * j >= P) break;  // no lane of the group holds pair j (uniform across the group)
      const int p = min(gl + G * j, P - 1);
      const uint64_t s = f2_fma(nth2, a2[j], s2[j]);  // the previous step's slack update
      s2[j] = s;
      const ulonglong2* row = reinterpret_cast<const ulonglong2*>(rows + (size_t)p * RS);
      uint64_t acc = 0ull;
#pragma unroll
      for (int q = 0; q < MAXD / 2; ++q) {
        if (2 * q < dim) {
          const ulonglong2 v = row[q];  // coordinates 2q and 2q + 1 of both faces
          acc = q == 0 ? f2_mul(v.x, dd[0]) : f2_fma(v.x, dd[2 * q], acc);
          if (2 * q + 1 < dim) acc = f2_fma(v.y, dd[2 * q + 1], acc);
        }
      }
      a2[j] = acc;
      float sa, sb, aa, ab;
      f2_unpack(s, &sa, &sb);
      f2_unpack(acc, &aa, &ab);
      theta_bound(sa, aa, tmin, tmax);
      theta_bound(sb, ab, tmin, tmax);
    }
    if constexpr (G <= 32) {
#pragma unroll
      for (int o = G / 2; o; o >>= 1) {
        tmin = fmaxf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o, G));
        tmax = fminf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o, G));
      }
    } else {
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        tmin = fmaxf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
        tmax = fminf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
      }
      float(*red)[2] = gs->red[step & 1];
      if ((gl & 31) == 0) {
        red[gl >> 5][0] = tmin;
        red[gl >> 5][1] = tmax;
      }
      group_bar(bar_id, G);
      tmin = red[0][0];
      tmax = red[0][1];
#pragma unroll
      for (int w = 1; w < G / 32; ++w) {
        tmin = fmaxf(tmin, red[w][0]);
        tmax = fminf(tmax, red[w][1]);
      }
    }
    if (isinf(tmax) || isinf(tmin) || tmax < tmin) ok = false;
    // this step's direction at the position coordinates the lane holds (coordinate k: block
    // k >> 2 on lane base + (k >> 2), half (k >> 1) & 1, cosine or sine k & 1)
    float dkl[XL];
#pragma unroll
    for (int r = 0; r < XL; ++r) {
      const int k = min(gl + G * r, MAXD - 1);
      if constexpr (G <= 32) {
        const int src = base + (k >> 2);
        const float va0 = __shfl_sync(0xffffffffu, c0a, src, G), va1 = __shfl_sync(0xffffffffu, c1a, src, G);
        const float vb0 = __shfl_sync(0xffffffffu, c0b, src, G), vb1 = __shfl_sync(0xffffffffu, c1b, src, G);
        dkl[r] = ((k >> 1) & 1) ? ((k & 1) ? vb1 : vb0) : ((k & 1) ? va1 : va0);
      } else {
        dkl[r] = gs->dir[batch & 1][t][k];
      }
    }
    nth = -0.0f;
    if (ok) {
      double th = __dadd_rn(__dmul_rn((double)ut, __dsub_rn(__dmul_rn(0.999999, (double)tmax), (double)tmin)),
                            (double)tmin);
      const float theta = __double2float_rn(th);
#pragma unroll
      for (int r = 0; r < XL; ++r)
        if (gl + G * r < dim) xl[r] = __fmaf_rn(theta, dkl[r], xl[r]);
      nth = -theta;
    }
    t = t + 1 == S ? 0 : t + 1;
  }
  return ok;
}

// Chains [first, last) of one region by the whole block (256 threads), G
// lanes per chain; groups past `last` repeat the last chain and store
// nothing, so every group takes the same number of trips (wide groups meet
// at named barriers 1 + group index). A failed chain stores `start`.
template <int MAXD, int G, int KP>
__device__ __forceinline__ void sample_chains_pairs(const float* __restrict__ rows, int P, int dim,
                                                    const float* __restrict__ start, int first, int last, int mixing,
                                                    uint32_t k0, uint32_t k1, uint32_t stream,
                                                    float* __restrict__ out, GroupScratch* gsa) {
  constexpr int XL = (MAXD + G - 1) / G;
  const int gl = threadIdx.x & (G - 1), gid = threadIdx.x / G, ngroups = blockDim.x / G;
  GroupScratch* gs = G > 32 ? gsa + gid : nullptr;
  for (int c0 = first; c0 < last; c0 += ngroups) {
    const int chain = c0 + gid;
    const int cc = chain < last ? chain : last - 1;
    float xl[XL];
#pragma unroll
    for (int r = 0; r < XL; ++r) {
      const int k = gl + G * r;
      xl[r] = k < dim ? start[k] : 0.f;
    }
    const bool ok = run_chain_pairs<MAXD, G, KP>(rows, P, dim, mixing, k0, k1, (uint32_t)cc, stream, xl, gl, gs,
                                                 1 + gid);
    if (chain < last) {
#pragma unroll
      for (int r = 0; r < XL; ++r) {
        const int k = gl + G * r;
        if (k < dim) out[(int64_t)chain * dim + k] = ok ? xl[r] : start[k];
      }
    }
  }
}

// The chains of one region with G lanes each (G from pair_group_width, one of
// 8 .. 256).
template <int MAXD, int KP>
__device__ __forceinline__ void sample_region(int G, const float* __restrict__ rows, int P, int dim,
                                              const float* __restrict__ start, int first, int last, int mixing,
                                              uint32_t k0, uint32_t k1, uint32_t stream, float* __restrict__ out,
                                              GroupScratch* gsa) {
  switch (G) {
    case 8:
      sample_chains_pairs<MAXD, 8, KP>(rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
      break;
    case 16:
      sample_chains_pairs<MAXD, 16, KP>(rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
      break;
    case 32:
      sample_chains_pairs<MAXD, 32, KP>(rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
      break;
    case 64:
      sample_chains_pairs<MAXD, 64, KP>(rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
      break;
    case 128:
      sample_chains_pairs<MAXD, 128, KP>(rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
      break;
    default:
      sample_chains_pairs<MAXD, 256, KP>(rows, P, dim, start, first, last, mixing, k0, k1, stream, out, gsa);
      break;
  }
}

// Copies P pair rows (stride floats each, 16-byte multiples) to shared memory.
__device__ __forceinline__ void stage_pairs(const float* __restrict__ rows, int P, int stride, float* sm) {
  const float4* src = reinterpret_cast<const float4*>(rows);
  float4* dst = reinterpret_cast<float4*>(sm);
  const int n = P * stride / 4;
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// Group width for `total` chains over `grid_warps` resident warps: 8 lanes
// per chain when there are enough chains to fill the grid that way, wider
// groups when there are few (the tail of an inflation).
__host__ __device__ __forceinline__ int group_width(int64_t total, int64_t grid_warps) {
  return total >= 8 * grid_warps ? 8 : total >= 4 * grid_warps ? 16 : 32;
}

}  // namespace csd
