// eizo_core.cuh -- EI-ZO stage bodies shared by the single-inflation kernels
// (eizo.cu) and the batched kernels (batch.cu): ordered compaction, the
// per-particle bisection and the greedy face placement.
#pragma once
#include <cfloat>

#include "check_core.cuh"
#include "sampler_core.cuh"

namespace csd {

struct EizoCounters {
  uint32_t total;     // colliding samples
  uint32_t first_m;   // colliding samples among the first M
  uint32_t placed;    // faces placed by the last faces_kernel
  int32_t status;     // 0 ok, 2 face capacity exceeded
};

// Ordered compaction of the colliding samples (first max_keep kept, in index
// order) and the first-M collision count; one block.
static __device__ __forceinline__ void compact_block(const uint8_t* __restrict__ flags,
                                                     const float* __restrict__ samples, int N, int M, int max_keep,
                                                     int dim, float* __restrict__ cols, EizoCounters* cnt) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t running;
  __shared__ uint32_t first_m;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) {
    running = 0;
    first_m = 0;
  }
  __syncthreads();
  for (int base = 0; base < N; base += blockDim.x) {
    int i = base + tid;
    uint32_t f = (i < N && !flags[i]) ? 1u : 0u;
    uint32_t ballot = __ballot_sync(0xffffffffu, f);
    uint32_t pre = __popc(ballot & ((1u << lane) - 1u));
    uint32_t fm = __popc(__ballot_sync(0xffffffffu, f && i < M));
    if (lane == 0) warp_sums[warp] = __popc(ballot);
    if (lane == 0 && fm) atomicAdd(&first_m, fm);
    __syncthreads();
    uint32_t off = 0;
    for (int w = 0; w < warp; ++w) off += warp_sums[w];
    uint32_t pos = running + off + pre;
    if (f && pos < (uint32_t)max_keep)
      for (int k = 0; k < dim; ++k) cols[(size_t)pos * dim + k] = samples[(size_t)i * dim + k];
    __syncthreads();
    if (tid == 0) {
      uint32_t tot = 0;
      for (int w = 0; w < nw; ++w) tot += warp_sums[w];
      running += tot;
    }
    __syncthreads();
  }
  if (tid == 0) {
    cnt->total = running;
    cnt->first_m = first_m;
  }
}


// One warp per particle: lane k holds coordinate k of the collision point,
// its projection and the bisection bounds; each step is a fused FK + check of
// the midpoint. Dot products are accumulated in coordinate order with
// fused multiply-adds (the order the CPU restatement uses).
template <bool SM>
static __device__ __forceinline__ void bisect_particle(const DevPlant& p, const WarpCtx<SM>& w, int i, int dim,
                                                       int steps, const float* __restrict__ ls,
                                                       const float* __restrict__ le, const VoxArgs& va,
                                                       float* __restrict__ cols, float* __restrict__ proj,
                                                       float* __restrict__ dist, int lane) {
  const float* ci = cols + (size_t)i * dim;
  // projection onto the segment (every lane evaluates the same serial sums)
  float seg2 = 0.f, a = 0.f;
  for (int k = 0; k < dim; ++k) {
    float dk = __fsub_rn(le[k], ls[k]);
    seg2 = __fmaf_rn(dk, dk, seg2);
    a = __fmaf_rn(__fsub_rn(ci[k], ls[k]), dk, a);
  }
  const float t = fminf(fmaxf(__fdiv_rn(a, seg2), 0.0f), 1.0f);
  const float omt = __fsub_rn(1.0f, t);
  float c = 0.f, pr = 0.f, lo = 0.f, hi = 0.f;
  if (lane < dim) {
    c = ci[lane];
    pr = __fmaf_rn(t, le[lane], __fmul_rn(omt, ls[lane]));
    lo = pr;
    hi = c;
  }
  for (int s = 0; s < steps; ++s) {
    const float mid = __fmul_rn(0.5f, __fadd_rn(lo, hi));
    __syncwarp();
    if (lane < dim) w.qs[lane] = mid;
    __syncwarp();
    fk_warp(p, w.qs, w.X, lane);
    const bool hit = check_config(p, w.stat, w.aabb, w.X, w.pose, lane, va);
    if (hit) {
      hi = mid;
      c = mid;
    } else {
      lo = mid;
    }
  }
  // distance to the projection, coordinates in order
  __syncwarp();
  if (lane < dim) w.qs[lane] = __fsub_rn(c, pr);
  __syncwarp();
  float s2 = 0.f;
  for (int k = 0; k < dim; ++k) s2 = __fmaf_rn(w.qs[k], w.qs[k], s2);
  if (lane < dim) {
    cols[(size_t)i * dim + lane] = c;
    proj[(size_t)i * dim + lane] = pr;
  }
  if (lane == 0) dist[i] = __fsqrt_rn(s2);
  __syncwarp();
}

// One block places up to max_faces faces (greedy, nearest collision first).
// rows (optional) receives each face as a face-pair row with its start slack
// at ls (put_face), the layout the EI-ZO sampler reads.
static __device__ __forceinline__ void faces_block(int K, int dim, int max_faces, int capacity, float margin,
                                                   const float* __restrict__ ls, const float* __restrict__ le,
                                                   const float* __restrict__ cols, const float* __restrict__ proj,
                                                   float* __restrict__ dist, float* __restrict__ A,
                                                   float* __restrict__ b, int* __restrict__ num_faces,
                                                   EizoCounters* cnt, float* __restrict__ rows = nullptr) {
  __shared__ float red_v[32];
  __shared__ int red_i[32];
  __shared__ float face[kMaxDim + 1];
  __shared__ int best_s;
  __shared__ float best_v;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  int nf = *num_faces;
  int placed = 0;
  int status = 0;
  for (; placed < max_faces; ++placed) {
    float bv = FLT_MAX;
    int bi = 0x7fffffff;
    for (int i = tid; i < K; i += blockDim.x) {
      float v = dist[i];
      if (v < bv || (v == bv && i < bi)) {
        bv = v;
        bi = i;
      }
    }
    for (int o = 16; o; o >>= 1) {
      float ov = __shfl_down_sync(0xffffffffu, bv, o);
      int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov < bv || (ov == bv && oi < bi)) {
        bv = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      red_v[warp] = bv;
      red_i[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      float v = FLT_MAX;
      int ix = 0x7fffffff;
      for (int w = 0; w < nw; ++w)
        if (red_v[w] < v || (red_v[w] == v && red_i[w] < ix)) {
          v = red_v[w];
          ix = red_i[w];
        }
      best_v = v;
      best_s = ix;
    }
    __syncthreads();
    if (!(best_v < FLT_MAX)) break;
    if (nf >= capacity) {
      status = 2;
      break;
    }
    if (tid == 0) {
      const int s = best_s;
      const float* c = cols + (size_t)s * dim;
      const float* pr = proj + (size_t)s * dim;
      float a[kMaxDim];
      float n2 = 0.f;
      for (int k = 0; k < dim; ++k) {
        a[k] = __fsub_rn(c[k], pr[k]);
        n2 = __fmaf_rn(a[k], a[k], n2);
      }
      float nrm = __fsqrt_rn(n2);
      for (int k = 0; k < dim; ++k) a[k] = __fdiv_rn(a[k], nrm);
      float bb = 0.f, v1 = 0.f, v2 = 0.f;
      for (int k = 0; k < dim; ++k) {
        bb = __fmaf_rn(a[k], c[k], bb);
        v1 = __fmaf_rn(a[k], ls[k], v1);
        v2 = __fmaf_rn(a[k], le[k], v2);
      }
      bb = __fsub_rn(bb, margin);
      v1 = __fsub_rn(v1, bb);
      v2 = __fsub_rn(v2, bb);
      float relax = v2 > v1 ? v2 : v1;
      relax = relax > 0 ? relax : 0;
      bb = __fadd_rn(bb, relax);
      for (int k = 0; k < dim; ++k) {
        A[(size_t)nf * dim + k] = a[k];
        face[k] = a[k];
      }
      if (rows) put_face(rows, dim, nf, a, bb, ls);
      b[nf] = bb;
      face[dim] = bb;
      dist[s] = FLT_MAX;
    }
    __syncthreads();
    const float bb = face[dim];
    for (int i = tid; i < K; i += blockDim.x) {
      if (dist[i] == FLT_MAX) continue;
      float v = 0.f;
      for (int k = 0; k < dim; ++k) v = __fmaf_rn(face[k], cols[(size_t)i * dim + k], v);
      if (__fsub_rn(v, bb) > 0.f) dist[i] = FLT_MAX;
    }
    ++nf;
    __syncthreads();
  }
  if (tid == 0) {
    *num_faces = nf;
    cnt->placed = (uint32_t)placed;
    cnt->status = status;
  }
}


}  // namespace csd
