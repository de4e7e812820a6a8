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

// The same chain run by a group of G lanes (G = 8, 16 or 32; 32 / G chains
// per warp). Jobs 0..ceil(dim/2)-1 are the Gaussian pairs and job ceil(dim/2)
// the theta uniform, each drawn from the Philox block and words the serial
// step_draws uses; lane gl of the group draws jobs gl, gl + G, ... and the
// direction is broadcast by shuffles. The group's lanes split the faces
// f = gl, gl + G, ...: each face's slack and A dir are accumulated in the
// serial order, and the theta bounds are max/min reductions, which do not
// depend on the order, so every chain ends bit for bit where run_chain ends.
// At is the face matrix transposed, At[k * stride + f], with the stride ST
// when ST > 0 (a shared-memory copy) and ldt otherwise. ROWS: At is instead a
// face-row copy (stage_rows: row f at At + f * ST, coordinates as float4
// vectors, b_f at coordinate MAXD) and bp is unused. x is replicated in
// the group's lanes. A chain whose line search fails keeps stepping without
// moving (so the groups of a warp stay convergent for the shuffles) and
// returns false.
template <int MAXD, int G, int ST, int U = 1, bool ROWS = false>
__device__ __forceinline__ bool run_chain_group(const float* __restrict__ At, int ldt, const float* __restrict__ bp,
                                                int F, int dim, int mixing, uint32_t k0, uint32_t k1,
                                                uint32_t chain, uint32_t stream, float* x, int gl) {
  static_assert(!ROWS || (ST > 0 && ST % 4 == 0 && MAXD % 4 == 0 && ST > MAXD), "face rows: float4 rows with b");
  constexpr int R = (MAXD / 2 + 1 + G - 1) / G;  // job rounds per lane
  const int stride = ST > 0 ? ST : ldt;
  const int npairs = (dim + 1) >> 1;
  bool ok = true;
  for (int step = 0; step < mixing; ++step) {
    float c0[R], c1[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      c0[r] = 0.f;
      c1[r] = 0.f;
      const int job = gl + r * G;
      if (job <= npairs) {
        const int word = 2 * job;
        uint32_t w[4];
        philox4x32_10((uint32_t)step, chain, stream, (uint32_t)(word >> 2), k0, k1, w);
        const uint32_t wa = (word & 2) ? w[2] : w[0];
        const uint32_t wb = (word & 2) ? w[3] : w[1];
        if (job < npairs) {
          float u = u01_open0(wa);
          float v = u01_open1(wb);
          float rad = __fsqrt_rn(__fmul_rn(-2.0f, log_unit(u)));
          float sn, cs;
          sincos_2pi(v, &sn, &cs);
          c0[r] = __fmul_rn(rad, cs);
          c1[r] = __fmul_rn(rad, sn);
        } else {
          c0[r] = u01_open0(wa);
        }
      }
    }
    float dir[MAXD];
#pragma unroll
    for (int k = 0; k < MAXD; ++k) {
      const int p = k >> 1;
      dir[k] = __shfl_sync(0xffffffffu, (k & 1) ? c1[p / G] : c0[p / G], p % G, G);
    }
    float utv = c0[0];
#pragma unroll
    for (int r = 1; r < R; ++r)
      if (npairs / G == r) utv = c0[r];
    const float ut = __shfl_sync(0xffffffffu, utv, npairs % G, G);
    float tmax = FLT_MAX, tmin = -FLT_MAX;
    // U faces per lane and trip (independent dot products for the scheduler)
    for (int f0 = gl; f0 < F; f0 += G * U) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int f = f0 + u * G;
        if (U == 1 || f < F) {
          float ax, ad, lb;
          if constexpr (ROWS) {
            // one 16-byte shared load per four coordinates
            const float4* row = reinterpret_cast<const float4*>(At + f * ST);
            float a[MAXD];
#pragma unroll
            for (int q = 0; q < MAXD / 4; ++q) {
              const float4 v = row[q];
              a[4 * q] = v.x;
              a[4 * q + 1] = v.y;
              a[4 * q + 2] = v.z;
              a[4 * q + 3] = v.w;
            }
            ax = __fmul_rn(a[0], x[0]);
            ad = __fmul_rn(a[0], dir[0]);
#pragma unroll
            for (int k = 1; k < MAXD; ++k) {
              if (k < dim) {
                ax = __fmaf_rn(a[k], x[k], ax);
                ad = __fmaf_rn(a[k], dir[k], ad);
              }
            }
            lb = __fsub_rn(At[f * ST + MAXD], ax);
          } else {
            const float* col = At + f;
            float a0 = col[0];
            ax = __fmul_rn(a0, x[0]);
            ad = __fmul_rn(a0, dir[0]);
#pragma unroll
            for (int k = 1; k < MAXD; ++k) {
              if (k < dim) {
                float ak = col[k * stride];
                ax = __fmaf_rn(ak, x[k], ax);
                ad = __fmaf_rn(ak, dir[k], ad);
              }
            }
            lb = __fsub_rn(bp[f], ax);
          }
          if (ad < 0.0f)
            tmin = fmaxf(tmin, __fdiv_rn(lb, ad));
          else if (ad > 0.0f)
            tmax = fminf(tmax, __fdiv_rn(lb, ad));
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o; o >>= 1) {
      tmin = fmaxf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o, G));
      tmax = fminf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o, G));
    }
    if (isinf(tmax) || isinf(tmin) || tmax < tmin) ok = false;
    if (ok) {
      double th = __dadd_rn(__dmul_rn((double)ut, __dsub_rn(__dmul_rn(0.999999, (double)tmax), (double)tmin)),
                            (double)tmin);
      float theta = __double2float_rn(th);
#pragma unroll
      for (int k = 0; k < MAXD; ++k)
        if (k < dim) x[k] = __fmaf_rn(theta, dir[k], x[k]);
    }
  }
  return ok;
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

// run_chain_group over a staged polytope (row stride ST, even; 8-byte aligned
// rows) with faces taken in adjacent pairs (f, f + 1), f even: one 64-bit
// shared-memory load brings coordinate k of both faces, and one packed FMA
// per dot product advances both. The configuration and the direction are
// kept duplicated in both halves ((x_k, x_k), (d_k, d_k)) so they pair with
// any face pair. Per face the operations and their order are those of
// run_chain_group (product, FMAs in coordinate order, b - A x, division), and
// the theta bounds are order-independent reductions, so the chain ends bit
// for bit where run_chain ends. U pairs per lane and trip.
template <int MAXD, int G, int ST, int U>
__device__ __forceinline__ bool run_chain_group_x2(const float* __restrict__ At, const float* __restrict__ bp, int F,
                                                   int dim, int mixing, uint32_t k0, uint32_t k1, uint32_t chain,
                                                   uint32_t stream, float* x, int gl) {
  static_assert(ST > 0 && ST % 2 == 0, "packed faces need an even staged stride");
  constexpr int R = (MAXD / 2 + 1 + G - 1) / G;
  const int npairs = (dim + 1) >> 1;
  uint64_t xx[MAXD];
#pragma unroll
  for (int k = 0; k < MAXD; ++k) xx[k] = f2_pack(x[k], x[k]);
  bool ok = true;
  for (int step = 0; step < mixing; ++step) {
    float c0[R], c1[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      c0[r] = 0.f;
      c1[r] = 0.f;
      const int job = gl + r * G;
      if (job <= npairs) {
        const int word = 2 * job;
        uint32_t w[4];
        philox4x32_10((uint32_t)step, chain, stream, (uint32_t)(word >> 2), k0, k1, w);
        const uint32_t wa = (word & 2) ? w[2] : w[0];
        const uint32_t wb = (word & 2) ? w[3] : w[1];
        if (job < npairs) {
          float u = u01_open0(wa);
          float v = u01_open1(wb);
          float rad = __fsqrt_rn(__fmul_rn(-2.0f, log_unit(u)));
          float sn, cs;
          sincos_2pi(v, &sn, &cs);
          c0[r] = __fmul_rn(rad, cs);
          c1[r] = __fmul_rn(rad, sn);
        } else {
          c0[r] = u01_open0(wa);
        }
      }
    }
    uint64_t dd[MAXD];
#pragma unroll
    for (int k = 0; k < MAXD; ++k) {
      const int p = k >> 1;
      const float dk = __shfl_sync(0xffffffffu, (k & 1) ? c1[p / G] : c0[p / G], p % G, G);
      dd[k] = f2_pack(dk, dk);
    }
    float utv = c0[0];
#pragma unroll
    for (int r = 1; r < R; ++r)
      if (npairs / G == r) utv = c0[r];
    const float ut = __shfl_sync(0xffffffffu, utv, npairs % G, G);
    float tmax = FLT_MAX, tmin = -FLT_MAX;
    for (int f0 = 2 * gl; f0 < F; f0 += 2 * G * U) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int f = f0 + 2 * G * u;
        if (U == 1 || f < F) {
          const float* col = At + f;
          uint64_t a = *reinterpret_cast<const uint64_t*>(col);
          uint64_t ax = f2_mul(a, xx[0]);
          uint64_t ad = f2_mul(a, dd[0]);
#pragma unroll
          for (int k = 1; k < MAXD; ++k) {
            if (k < dim) {
              a = *reinterpret_cast<const uint64_t*>(col + k * ST);
              ax = f2_fma(a, xx[k], ax);
              ad = f2_fma(a, dd[k], ad);
            }
          }
          const uint64_t lb2 = f2_sub(*reinterpret_cast<const uint64_t*>(bp + f), ax);
          float lb0, lb1, ad0, ad1;
          f2_unpack(lb2, &lb0, &lb1);
          f2_unpack(ad, &ad0, &ad1);
          if (ad0 < 0.0f)
            tmin = fmaxf(tmin, __fdiv_rn(lb0, ad0));
          else if (ad0 > 0.0f)
            tmax = fminf(tmax, __fdiv_rn(lb0, ad0));
          if (f + 1 < F) {  // the pair's second face (row entries past F are never used)
            if (ad1 < 0.0f)
              tmin = fmaxf(tmin, __fdiv_rn(lb1, ad1));
            else if (ad1 > 0.0f)
              tmax = fminf(tmax, __fdiv_rn(lb1, ad1));
          }
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o; o >>= 1) {
      tmin = fmaxf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o, G));
      tmax = fminf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o, G));
    }
    if (isinf(tmax) || isinf(tmin) || tmax < tmin) ok = false;
    if (ok) {
      double th = __dadd_rn(__dmul_rn((double)ut, __dsub_rn(__dmul_rn(0.999999, (double)tmax), (double)tmin)),
                            (double)tmin);
      const float theta = __double2float_rn(th);
      const uint64_t tt = f2_pack(theta, theta);
#pragma unroll
      for (int k = 0; k < MAXD; ++k)
        if (k < dim) xx[k] = f2_fma(tt, dd[k], xx[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < MAXD; ++k) {
    float lo, hi;
    f2_unpack(xx[k], &lo, &hi);
    x[k] = lo;
  }
  return ok;
}

// Writes coordinates gl, gl + G, ... of a group-replicated vector.
template <int MAXD, int G>
__device__ __forceinline__ void group_store(const float* x, int dim, int gl, float* __restrict__ dst, bool ok,
                                            const float* __restrict__ fallback) {
#pragma unroll
  for (int r = 0; r < (MAXD + G - 1) / G; ++r) {
    const int k = gl + r * G;
    float v = 0.f;
#pragma unroll
    for (int j = 0; j < MAXD; ++j)
      if (j == k) v = x[j];
    if (k < dim) dst[k] = ok ? v : fallback[k];
  }
}

// Shared-memory staging of one polytope for the group sampler: rows
// k < dim of At at stride ST, then b at row MAXD. Sized (MAXD + 1) * ST floats.
constexpr int kStageFaces8 = 2048;   // faces staged for dim <= 8
constexpr int kStageFaces16 = 1024;  // faces staged for dim <= 16
constexpr size_t kStageBytes = 9 * kStageFaces8 * sizeof(float);
static_assert(9 * kStageFaces8 >= 17 * kStageFaces16, "staging buffer");

// Staging capacity of a kernel with MINB resident blocks per SM: the largest
// buffer that MINB blocks fit in the SM's 227 KB (2 blocks: 3072 / 1536
// faces, 3 blocks: 2048 / 1024, 4 blocks: 1536 / 768).
// Face-row staging (stage_rows): row f holds a_f0 .. a_f(MAXD-1) (zero past
// dim) and b_f at MAXD, kRowStride floats apart. The strides are multiples of
// 16 bytes for the float4 loads, and 12 and 20 floats put the eight rows a
// group reads at once in eight disjoint sets of four banks.
template <int MAXD>
constexpr int kRowStride = MAXD <= 8 ? 12 : 20;

template <int MINB>
struct StageCfg {
  static constexpr int f8 = MINB <= 2 ? 3072 : MINB == 3 ? 2048 : 1536;
  static constexpr int f16 = f8 / 2;
  static constexpr size_t bytes = 9 * (size_t)f8 * sizeof(float);
  // faces the same buffer holds as face rows
  static constexpr int r8 = (int)(bytes / (kRowStride<8> * sizeof(float)));
  static constexpr int r16 = (int)(bytes / (kRowStride<16> * sizeof(float)));
  static_assert(9 * f8 >= 17 * f16, "staging buffer");
  static_assert(MINB * bytes <= 227 * 1024, "MINB staging buffers fit one SM");
};

template <int MAXD, int ST>
__device__ __forceinline__ void stage_polytope(const float* __restrict__ At, int ldt, const float* __restrict__ b,
                                               int F, int dim, float* sm) {
  for (int i = threadIdx.x; i < dim * F; i += blockDim.x) {
    const int k = i / F, f = i - k * F;
    sm[k * ST + f] = At[(int64_t)k * ldt + f];
  }
  for (int f = threadIdx.x; f < F; f += blockDim.x) sm[MAXD * ST + f] = b[f];
}

// Stages F faces of a transposed polytope (At[k * ldt + f], b[f]) as face
// rows: F * kRowStride<MAXD> floats of sm (16-byte aligned).
template <int MAXD>
__device__ __forceinline__ void stage_rows(const float* __restrict__ At, int ldt, const float* __restrict__ b, int F,
                                           int dim, float* sm) {
  constexpr int RS = kRowStride<MAXD>;
  for (int i = threadIdx.x; i < MAXD * F; i += blockDim.x) {
    const int k = i / F, f = i - k * F;
    sm[f * RS + k] = k < dim ? At[(int64_t)k * ldt + f] : 0.f;
  }
  for (int f = threadIdx.x; f < F; f += blockDim.x) sm[f * RS + MAXD] = b[f];
}

// Staged layouts of the group sampler: transposed columns, transposed columns
// read in packed face pairs, face rows.
enum : int { kLayStrided = 0, kLayPacked = 1, kLayRows = 2 };

// Chains [first, last) of one polytope by the whole block, G lanes per
// chain; the trip count is uniform across the block (groups past `last`
// repeat the last chain and store nothing). A failed chain stores `start`.
template <int MAXD, int G, int ST, int U, int LAY = kLayStrided>
__device__ __forceinline__ void sample_chains(const float* __restrict__ At, int ldt, const float* __restrict__ b,
                                              int F, int dim, const float* __restrict__ start, int first, int last,
                                              int mixing, uint32_t k0, uint32_t k1, uint32_t stream,
                                              float* __restrict__ out) {
  const int lane = threadIdx.x & 31, gl = lane & (G - 1);
  const int gid = (threadIdx.x >> 5) * (32 / G) + lane / G;
  const int ngroups = (blockDim.x >> 5) * (32 / G);
  for (int c0 = first; c0 < last; c0 += ngroups) {
    const int chain = c0 + gid;
    const int cc = chain < last ? chain : last - 1;
    float x[MAXD];
#pragma unroll
    for (int k = 0; k < MAXD; ++k) x[k] = k < dim ? start[k] : 0.f;
    bool ok;
    if constexpr (LAY == kLayPacked && ST > 0)
      ok = run_chain_group_x2<MAXD, G, ST, U>(At, b, F, dim, mixing, k0, k1, (uint32_t)cc, stream, x, gl);
    else
      ok = run_chain_group<MAXD, G, ST, U, LAY == kLayRows>(At, ldt, b, F, dim, mixing, k0, k1, (uint32_t)cc, stream,
                                                           x, gl);
    if (chain < last) group_store<MAXD, G>(x, dim, gl, out + (int64_t)chain * dim, ok, start);
  }
}

// Group width for `total` chains over `grid_warps` resident warps: 8 lanes
// per chain when there are enough chains to fill the grid that way, wider
// groups when there are few (the tail of an inflation).
__host__ __device__ __forceinline__ int group_width(int64_t total, int64_t grid_warps) {
  return total >= 8 * grid_warps ? 8 : total >= 4 * grid_warps ? 16 : 32;
}

// One polytope's chains [first, last) read from `sm` when `staged` (the caller
// staged it: by stage_rows for LAY == kLayRows, else by stage_polytope with
// strides ST8 / ST16), else from global memory.
// kLayPacked: the staged path takes faces in packed pairs (U pairs per trip).
template <int MAXD, int U, int LAY = kLayStrided, int ST8 = kStageFaces8, int ST16 = kStageFaces16>
__device__ __forceinline__ void sample_range(const float* __restrict__ At, int ldt, const float* __restrict__ b,
                                             int F, int dim, const float* __restrict__ start, int first, int last,
                                             int mixing, uint32_t k0, uint32_t k1, uint32_t stream,
                                             float* __restrict__ out, int G, float* sm, bool staged) {
  constexpr int ST = LAY == kLayRows ? kRowStride<MAXD> : MAXD <= 8 ? ST8 : ST16;
  if (staged) {
    const float* sAt = sm;
    const float* sb = LAY == kLayRows ? nullptr : sm + MAXD * ST;
    if (G == 8)
      sample_chains<MAXD, 8, ST, U, LAY>(sAt, ST, sb, F, dim, start, first, last, mixing, k0, k1, stream, out);
    else if (G == 16)
      sample_chains<MAXD, 16, ST, U, LAY>(sAt, ST, sb, F, dim, start, first, last, mixing, k0, k1, stream, out);
    else
      sample_chains<MAXD, 32, ST, U, LAY>(sAt, ST, sb, F, dim, start, first, last, mixing, k0, k1, stream, out);
  } else {
    if (G == 8)
      sample_chains<MAXD, 8, 0, U>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out);
    else if (G == 16)
      sample_chains<MAXD, 16, 0, U>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out);
    else
      sample_chains<MAXD, 32, 0, U>(At, ldt, b, F, dim, start, first, last, mixing, k0, k1, stream, out);
  }
}

}  // namespace csd
