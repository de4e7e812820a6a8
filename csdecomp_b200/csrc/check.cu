// check.cu -- fused forward kinematics + collision checks on sm_100a.
//
// Reference pipeline (per call): executeForwardKinematicsKernel writes every
// link transform of every configuration to HBM (cuda_forward_kinematics.cu:59-90),
// pairCollisionFreeKernel runs one thread per (configuration, pair) and
// re-multiplies two 4x4 transforms per pair (cuda_collision_checker.cu:16-64),
// and poolPairCollisionFreeResultsKernel ANDs the N*P byte flags (:66-85).
//
// Here one warp checks one configuration end to end (check_core.cuh): FK,
// placement and the pair sweep stay in registers and shared memory, the
// static geometry is staged into shared memory once per block, and a warp
// vote stops the sweep at the first colliding pair. Only the configurations
// and the verdict bytes touch HBM.
#include <algorithm>

#include "check_core.cuh"

namespace csd {

template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) check_points_kernel(DevPlant p, const float* __restrict__ q,
                                                                          int64_t n, VoxArgs va,
                                                                          uint8_t* __restrict__ out) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  const WarpCtx<SM> w = warp_setup<SM>(p, smem4, &bar);
  if (!w.ok) return;
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nw) {
    if (lane < p.dim) w.qs[lane] = q[i * p.dim + lane];
    __syncwarp();
    fk_warp(p, w.qs, w.X, lane);
    const bool hit = check_config(p, w.stat, w.aabb, w.X, w.pose, lane, va);
    if (lane == 0) out[i] = hit ? 0 : 1;
  }
}

// ------------------------------------------------------------------ edges
__device__ __forceinline__ int64_t edge_points(const float* q1, const float* q2, int d, float step, int mode) {
  if (mode == CSD_EDGE_LINF) {
    float m = 0.f;
    for (int k = 0; k < d; ++k) m = fmaxf(m, fabsf(__fsub_rn(q2[k], q1[k])));
    return (int64_t)ceilf(__fdiv_rn(m, step)) + 1;
  }
  float s = 0.f;
  for (int k = 0; k < d; ++k) {
    float x = __fsub_rn(q2[k], q1[k]);
    s = __fadd_rn(s, __fmul_rn(x, x));
  }
  float nrm = __fsqrt_rn(s);
  if (mode == CSD_EDGE_L2_REF) return (int64_t)ceilf(__fdiv_rn(nrm, step));
  float x = __fadd_rn(__fdiv_rn(nrm, step), 2.0f);
  return (int64_t)(uint32_t)x;
}

__device__ __forceinline__ void lerp_point(const float* q1, const float* q2, int d, float t, float* out) {
  float omt = __fsub_rn(1.0f, t);
  for (int k = 0; k < d; ++k) out[k] = __fadd_rn(__fmul_rn(t, q2[k]), __fmul_rn(omt, q1[k]));
}

// Coordinate of point k of an edge from its endpoint coordinates (a1, a2),
// under a discretisation rule (see csd_capi.h).
__device__ __forceinline__ float edge_coord(float a1, float a2, int64_t np, int mode, int64_t k) {
  float t;
  if (mode == CSD_EDGE_L2_REF) {
    t = __double2float_rn(__ddiv_rn((double)k, (double)np));
  } else if (mode == CSD_EDGE_LINF) {
    if (np - 1 == 0) return a1;
    t = __double2float_rn(__ddiv_rn((double)k, (double)(np - 1)));
  } else {
    if (k == 0) return a1;
    if (k == 1) return a2;
    t = __fmul_rn(__double2float_rn(__ddiv_rn(1.0, (double)(np - 1))), (float)(k - 1));
  }
  return __fadd_rn(__fmul_rn(t, a2), __fmul_rn(__fsub_rn(1.0f, t), a1));
}

// Point k of an edge under a discretisation rule (see csd_capi.h).
__device__ __forceinline__ void edge_point(const float* q1, const float* q2, int d, int64_t np, int mode, int64_t k,
                                           float* out) {
  if (mode == CSD_EDGE_L2_REF) {
    float t = __double2float_rn(__ddiv_rn((double)k, (double)np));
    lerp_point(q1, q2, d, t, out);
  } else if (mode == CSD_EDGE_LINF) {
    int64_t T = np - 1;
    if (T == 0) {
      for (int i = 0; i < d; ++i) out[i] = q1[i];
    } else {
      float t = __double2float_rn(__ddiv_rn((double)k, (double)T));
      lerp_point(q1, q2, d, t, out);
    }
  } else {
    if (k == 0) {
      for (int i = 0; i < d; ++i) out[i] = q1[i];
    } else if (k == 1) {
      for (int i = 0; i < d; ++i) out[i] = q2[i];
    } else {
      float ts = __double2float_rn(__ddiv_rn(1.0, (double)(np - 1)));
      lerp_point(q1, q2, d, __fmul_rn(ts, (float)(k - 1)), out);
    }
  }
}

// One warp per edge, edges taken from a work counter. Points are visited
// coarse to fine: with G = ceil(n/32), the visit order is g, G+g, 2G+g, ...
// for g = 0, 1, ..., so the first 32 visits sample the whole edge evenly.
// Pair index e of the upper triangle (i < j, row-major) of n nodes -> (i, j):
// e = i n - i (i + 1) / 2 + (j - i - 1). The double-precision estimate of i
// is corrected with exact integer row starts.
static __device__ __forceinline__ void edge_pair(int64_t e, int64_t n, int64_t* i, int64_t* j) {
  auto row_start = [n](int64_t r) { return r * n - r * (r + 1) / 2; };
  const double b = 2.0 * (double)n - 1.0;
  int64_t r = (int64_t)floor((b - sqrt(b * b - 8.0 * (double)e)) * 0.5);
  r = r < 0 ? 0 : r > n - 2 ? n - 2 : r;
  while (r > 0 && row_start(r) > e) --r;
  while (r < n - 2 && row_start(r + 1) <= e) ++r;
  *i = r;
  *j = e - row_start(r) + r + 1;
}

// nodes > 0: the edges are every pair i < j of the `nodes` configurations in
// `starts` (ends unused), in upper-triangle row-major order.
template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) check_edges_kernel(DevPlant p, const float* __restrict__ starts,
                                                                         const float* __restrict__ ends, int64_t n,
                                                                         float step, int mode,
                                                                         uint8_t* __restrict__ out,
                                                                         int64_t* __restrict__ pts,
                                                                         unsigned long long* counter, int64_t nodes) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  const WarpCtx<SM> w = warp_setup<SM>(p, smem4, &bar);
  if (!w.ok) return;
  const int lane = threadIdx.x & 31;
  const int d = p.dim;
  VoxArgs none{nullptr, 0, 0.f, nullptr, nullptr, 0};
  while (true) {
    unsigned long long e = 0;
    if (lane == 0) e = atomicAdd(counter, 1ull);
    e = __shfl_sync(kFull, e, 0);
    if (e >= (unsigned long long)n) break;
    __syncwarp();
    if (nodes > 0) {
      int64_t i = 0, j = 0;
      edge_pair((int64_t)e, nodes, &i, &j);
      if (lane < d) {
        w.q1[lane] = starts[i * d + lane];
        w.q2[lane] = starts[j * d + lane];
      }
    } else if (lane < d) {
      w.q1[lane] = starts[e * d + lane];
      w.q2[lane] = ends[e * d + lane];
    }
    __syncwarp();
    const int64_t np = edge_points(w.q1, w.q2, d, step, mode);
    const int64_t G = (np + 31) / 32;
    bool collided = false;
    int64_t checked = 0;
    const float a1 = lane < d ? w.q1[lane] : 0.f, a2 = lane < d ? w.q2[lane] : 0.f;
    for (int64_t v = 0; v < 32 * G && !collided; ++v) {
      const int64_t k = (v % 32) * G + v / 32;
      if (k >= np) continue;
      const float x = edge_coord(a1, a2, np, mode, k);
      __syncwarp();
      if (lane < d) w.qs[lane] = x;
      __syncwarp();
      fk_warp(p, w.qs, w.X, lane);
      ++checked;
      collided = check_config(p, w.stat, w.aabb, w.X, w.pose, lane, none);
    }
    if (lane == 0) {
      out[e] = collided ? 0 : 1;
      if (pts) pts[e] = checked;
    }
  }
}

// ------------------------------------------------- surrogate-ranked edge checks
// Points per edge (thread per edge).
__global__ void edge_count_kernel(const float* __restrict__ s, const float* __restrict__ e, int64_t n, int d,
                                  float step, int mode, int64_t* __restrict__ counts) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    counts[i] = edge_points(s + i * d, e + i * d, d, step, mode);
}

// The points of edges [e0, e1) as rows of x (edge i's points from row
// off[i] - off[e0]); warp per edge, lane per point.
__global__ void edge_materialize_kernel(const float* __restrict__ s, const float* __restrict__ e, int64_t e0,
                                        int64_t e1, const int64_t* __restrict__ off, int d, int mode,
                                        float* __restrict__ x) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = e0 + blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < e1; i += nw) {
    const int64_t np = off[i + 1] - off[i];
    float* xi = x + (off[i] - off[e0]) * d;
    for (int64_t k = lane; k < np; k += 32)
      for (int c = 0; c < d; ++c) xi[k * d + c] = edge_coord(s[i * d + c], e[i * d + c], np, mode, k);
  }
}

// Warp per edge of [e0, e1): if logits are given, the point with the highest
// logit in each residue class k mod 32 is a candidate, the candidates are
// checked in decreasing logit (at most `top`), then every other point
// coarse-to-fine as check_edges_kernel visits them. The verdict is the AND
// over all points either way; only the order (and so the early exit) depends
// on the logits.
template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3)
    check_edges_ranked_kernel(DevPlant p, const float* __restrict__ starts, const float* __restrict__ ends, int64_t e0,
                              int64_t e1, const int64_t* __restrict__ off, const float* __restrict__ logits, int top,
                              int mode, uint8_t* __restrict__ out, int64_t* __restrict__ pts,
                              unsigned long long* counter) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  const WarpCtx<SM> w = warp_setup<SM>(p, smem4, &bar);
  if (!w.ok) return;
  const int lane = threadIdx.x & 31;
  const int d = p.dim;
  VoxArgs none{};
  while (true) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(counter, 1ull);
    c = __shfl_sync(kFull, c, 0);
    const int64_t e = e0 + (int64_t)c;
    if (e >= e1) break;
    const int64_t np = off[e + 1] - off[e];
    const float a1 = lane < d ? starts[e * d + lane] : 0.f, a2 = lane < d ? ends[e * d + lane] : 0.f;
    bool collided = false;
    int64_t checked = 0;
    // candidates: best logit of each residue class, sorted descending across the warp
    float bv = -FLT_MAX;
    int64_t bk = -1;
    if (logits) {
      const float* lg = logits + (off[e] - off[e0]);
      for (int64_t k = lane; k < np; k += 32) {
        const float v = lg[k];
        if (v > bv || bk < 0) {
          bv = v;
          bk = k;
        }
      }
    }
    // bitonic sort of (bv, bk) over the 32 lanes: lane r ends with the r-th
    // candidate by decreasing logit (lower index on ties; empty classes last)
    auto before = [](float va, int64_t ka, float vb, int64_t kb) {
      return ka >= 0 && (kb < 0 || va > vb || (va == vb && ka < kb));
    };
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const float ov = __shfl_xor_sync(kFull, bv, stride);
        const int64_t ok = __shfl_xor_sync(kFull, bk, stride);
        const bool descending = (lane & size) == 0;
        const bool lower = (lane & stride) == 0;
        const bool take = (lower == descending) ? before(ov, ok, bv, bk) : before(bv, bk, ov, ok);
        if (take) {
          bv = ov;
          bk = ok;
        }
      }
    }
    int ncand = logits ? min(top, np < 32 ? (int)np : 32) : 0;
    const int64_t G = (np + 31) / 32;
    // one visiting loop (one inlined check): candidates r < ncand first, then coarse-to-fine
    int r = 0;
    int64_t v = 0;
    while (!collided) {
      int64_t k;
      if (r < ncand) {
        k = __shfl_sync(kFull, bk, r);
        ++r;
        if (k < 0) {  // fewer candidates than `top`: the rest are empty classes
          ncand = r - 1;
          continue;
        }
      } else {
        if (v >= 32 * G) break;
        k = (v % 32) * G + v / 32;
        ++v;
        if (k >= np) continue;
        if (__any_sync(kFull, lane < ncand && bk == k)) continue;  // checked as a candidate
      }
      const float x = edge_coord(a1, a2, np, mode, k);
      __syncwarp();
      if (lane < d) w.qs[lane] = x;
      __syncwarp();
      fk_warp(p, w.qs, w.X, lane);
      ++checked;
      collided = check_config(p, w.stat, w.aabb, w.X, w.pose, lane, none);
    }
    if (lane == 0) {
      out[e] = collided ? 0 : 1;
      if (pts) pts[e] = checked;
    }
  }
}

// ---------------------------------------------------------------- FK output
// Warp per configuration; lane l writes reference link l's 4x4 (column-major).
__global__ void __launch_bounds__(32 * kWarpsPerBlock) fk_kernel(DevPlant p, const float* __restrict__ q, int64_t n,
                                                                float* __restrict__ tf_out) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  const WarpCtx<false> w = warp_setup<false>(p, smem4, &bar);
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nw) {
    if (lane < p.dim) w.qs[lane] = q[i * p.dim + lane];
    __syncwarp();
    fk_warp(p, w.qs, w.X, lane);
    __syncwarp();
    for (int l = lane; l < p.num_links; l += kWarp) {
      const int s = __ldg(p.link_slot + l);
      const float* F = p.link_fixed + 12 * l;
      float Rf[9], tfx[3], R[9], t[3];
      for (int k = 0; k < 9; ++k) Rf[k] = __ldg(F + k);
      for (int k = 0; k < 3; ++k) tfx[k] = __ldg(F + 9 + k);
      if (s == -2) {
        for (int k = 0; k < 9; ++k) R[k] = 0.f;
        for (int k = 0; k < 3; ++k) t[k] = 0.f;
      } else if (s == -1) {
        for (int k = 0; k < 9; ++k) R[k] = Rf[k];
        for (int k = 0; k < 3; ++k) t[k] = tfx[k];
      } else {
        const float* src = w.X + s * 12;
        compose(src, src + 9, Rf, tfx, R, t);
      }
      float4* dst = reinterpret_cast<float4*>(tf_out + (i * p.num_links + l) * 16);
      const float last = s == -2 ? 0.f : 1.f;
      dst[0] = make_float4(R[0], R[1], R[2], 0.f);
      dst[1] = make_float4(R[3], R[4], R[5], 0.f);
      dst[2] = make_float4(R[6], R[7], R[8], 0.f);
      dst[3] = make_float4(t[0], t[1], t[2], last);
    }
    __syncwarp();
  }
}

// Single pair on the device (one thread), GPU contact rule.
__global__ void pair_kernel(int ta, const float* g, int tb, uint8_t* out) {
  // g: [2][16] world-format poses computed on the host from FP32 inputs
  *out = pair_hit(ta, g, tb, g + 16) ? 0 : 1;
}

// ----------------------------------------------------------------- launchers
template <typename K>
static csd_status_t launch_grid(const csd_plant_s* p, K kernel, bool sm, int64_t work_warps, size_t* smem, int* grid) {
  *smem = (size_t)warp_floats(p->dp) * sizeof(float) * kWarpsPerBlock + (sm ? (size_t)p->dp.static_bytes : 0);
  return grid_for(kernel, *smem, work_warps, grid, kWarpsPerBlock);
}

csd_status_t launch_check_points(const csd_plant_s* p, const float* q, int64_t n, const VoxelTables& vt,
                                 uint8_t* out, cudaStream_t st) {
  if (n <= 0) return CSD_OK;
  const VoxArgs va = vox_args(vt);
  size_t smem = 0;
  int grid = 0;
  csd_status_t s;
  if (statics_in_smem(p)) {
    if ((s = launch_grid(p, check_points_kernel<true>, true, n, &smem, &grid))) return s;
    check_points_kernel<true><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, q, n, va, out);
  } else {
    if ((s = launch_grid(p, check_points_kernel<false>, false, n, &smem, &grid))) return s;
    check_points_kernel<false><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, q, n, va, out);
  }
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_fk(const csd_plant_s* p, const float* q, int64_t n, float* tf, cudaStream_t st) {
  if (n <= 0) return CSD_OK;
  size_t smem = 0;
  int grid = 0;
  csd_status_t s = launch_grid(p, fk_kernel, false, n, &smem, &grid);
  if (s) return s;
  fk_kernel<<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, q, n, tf);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_edge_count(const float* s, const float* e, int64_t n, int d, float step, int mode,
                               int64_t* counts, cudaStream_t st) {
  if (n <= 0) return CSD_OK;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 8 * device_sm_count());
  edge_count_kernel<<<grid, 256, 0, st>>>(s, e, n, d, step, mode, counts);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_edge_materialize(const float* s, const float* e, int64_t e0, int64_t e1, const int64_t* off, int d,
                                     int mode, float* x, cudaStream_t st) {
  if (e1 <= e0) return CSD_OK;
  const int grid = (int)std::min<int64_t>((e1 - e0 + 7) / 8, 8 * device_sm_count());
  edge_materialize_kernel<<<grid, 256, 0, st>>>(s, e, e0, e1, off, d, mode, x);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_check_edges_ranked(const csd_plant_s* p, const float* s0, const float* e0p, int64_t e0, int64_t e1,
                                       const int64_t* off, const float* logits, int top, int mode, uint8_t* out,
                                       int64_t* pts, unsigned int* counter, cudaStream_t st) {
  if (e1 <= e0) return CSD_OK;
  size_t smem = 0;
  int grid = 0;
  csd_status_t s;
  CSD_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(counter);
  if (statics_in_smem(p)) {
    if ((s = launch_grid(p, check_edges_ranked_kernel<true>, true, e1 - e0, &smem, &grid))) return s;
    check_edges_ranked_kernel<true><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, s0, e0p, e0, e1, off, logits, top,
                                                                              mode, out, pts, ctr);
  } else {
    if ((s = launch_grid(p, check_edges_ranked_kernel<false>, false, e1 - e0, &smem, &grid))) return s;
    check_edges_ranked_kernel<false><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, s0, e0p, e0, e1, off, logits,
                                                                               top, mode, out, pts, ctr);
  }
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_check_edges(const csd_plant_s* p, const float* s0, const float* e0, int64_t n, float step,
                                int mode, uint8_t* out, int64_t* pts, unsigned int* counter, cudaStream_t st,
                                int64_t nodes) {
  if (n <= 0) return CSD_OK;
  size_t smem = 0;
  int grid = 0;
  csd_status_t s;
  CSD_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(counter);
  if (statics_in_smem(p)) {
    if ((s = launch_grid(p, check_edges_kernel<true>, true, n, &smem, &grid))) return s;
    check_edges_kernel<true><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, s0, e0, n, step, mode, out, pts, ctr,
                                                                       nodes);
  } else {
    if ((s = launch_grid(p, check_edges_kernel<false>, false, n, &smem, &grid))) return s;
    check_edges_kernel<false><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, s0, e0, n, step, mode, out, pts, ctr,
                                                                        nodes);
  }
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_pair(int ta, const float* g_dev, int tb, uint8_t* out, cudaStream_t st) {
  pair_kernel<<<1, 1, 0, st>>>(ta, g_dev, tb, out);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

}  // namespace csd
