// check.cu -- fused forward kinematics + collision checks on sm_100a.
//
// Reference pipeline (per call): executeForwardKinematicsKernel writes every
// link transform of every configuration to HBM (cuda_forward_kinematics.cu:59-90),
// pairCollisionFreeKernel runs one thread per (configuration, pair) and
// re-multiplies two 4x4 transforms per pair (cuda_collision_checker.cu:16-64),
// and poolPairCollisionFreeResultsKernel ANDs the N*P byte flags (:66-85).
//
// Here one warp owns a batch of 32 configurations:
//   1. FK, lane = configuration: each lane walks the moving joints of its own
//      configuration and leaves 3x4 slot transforms in shared memory
//      ([slot][12][33] floats: the 33-float row stride keeps both the
//      lane-contiguous writes and the per-slot reads of step 2 conflict free).
//   2. For each configuration of the batch in turn, lane = geometry: the warp
//      places the moving geometries (world poses to shared memory), then
//      sweeps the pairs: a lane holds one moving sphere and all lanes stream
//      the same static geometry (a broadcast load), then the remaining pairs
//      are split across lanes. A warp vote after every few static geometries
//      stops the sweep at the first colliding pair.
// Nothing but the input configurations and the verdicts touches HBM.
#include <algorithm>

#include "check_core.cuh"

namespace csd {

__global__ void __launch_bounds__(128) check_points_kernel(DevPlant p, const float* __restrict__ q, int64_t n,
                                                           VoxArgs va, uint8_t* __restrict__ out) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tf = smem + warp * per_warp_floats(p);
  float* qbuf = warp_qbuf(p, tf);
  float* pose = warp_pose(p, tf);
  const int64_t nbatch = (n + 31) / 32;
  for (int64_t b = (int64_t)blockIdx.x * wpb + warp; b < nbatch; b += (int64_t)gridDim.x * wpb) {
    const int64_t base = b * 32;
    const int cnt = (int)(n - base < 32 ? n - base : 32);
    // stage the batch's configurations (coalesced) into [k][lane]
    for (int w = lane; w < cnt * p.dim; w += 32) {
      int c = w / p.dim, k = w - c * p.dim;
      qbuf[k * kRow + c] = q[base * p.dim + w];
    }
    __syncwarp();
    if (lane < cnt) fk_lane(p, qbuf, tf, lane);
    __syncwarp();
    uint8_t verdict = 0;
    for (int c = 0; c < cnt; ++c) {
      bool hit = check_config(p, tf, pose, c, lane, va);
      if (lane == c) verdict = hit ? 0 : 1;
    }
    if (lane < cnt) out[base + lane] = verdict;
    __syncwarp();
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
// coarse to fine: batch g holds points g, G+g, 2G+g, ... (G = ceil(n/32)), so
// the first batch already samples the whole edge at 32 even spacings.
__global__ void __launch_bounds__(128) check_edges_kernel(DevPlant p, const float* __restrict__ starts,
                                                          const float* __restrict__ ends, int64_t n, float step,
                                                          int mode, uint8_t* __restrict__ out,
                                                          int64_t* __restrict__ pts, unsigned long long* counter) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tf = smem + warp * per_warp_floats(p);
  float* qbuf = warp_qbuf(p, tf);
  float* pose = warp_pose(p, tf);
  const int d = p.dim;
  VoxArgs none{nullptr, 0, 0.f, nullptr, nullptr, 0};
  while (true) {
    unsigned long long e = 0;
    if (lane == 0) e = atomicAdd(counter, 1ull);
    e = __shfl_sync(kFull, e, 0);
    if (e >= (unsigned long long)n) break;
    float q1[kMaxDim], q2[kMaxDim];
    for (int k = 0; k < d; ++k) {
      q1[k] = starts[e * d + k];
      q2[k] = ends[e * d + k];
    }
    const int64_t np = edge_points(q1, q2, d, step, mode);
    const int64_t G = (np + 31) / 32;
    bool collided = false;
    int64_t checked = 0;
    for (int64_t g = 0; g < G && !collided; ++g) {
      const int64_t k = (int64_t)lane * G + g;
      if (k < np) {
        float qk[kMaxDim];
        edge_point(q1, q2, d, np, mode, k, qk);
        for (int i = 0; i < d; ++i) qbuf[i * kRow + lane] = qk[i];
        fk_lane(p, qbuf, tf, lane);
      }
      __syncwarp();
      for (int c = 0; c < 32; ++c) {
        if ((int64_t)c * G + g >= np) continue;
        ++checked;
        if (check_config(p, tf, pose, c, lane, none)) {
          collided = true;
          break;
        }
      }
      __syncwarp();
    }
    if (lane == 0) {
      out[e] = collided ? 0 : 1;
      if (pts) pts[e] = checked;
    }
  }
}

// ---------------------------------------------------------------- FK output
// Lane = configuration; transforms of all reference links as 4x4 column-major.
__global__ void __launch_bounds__(128) fk_kernel(DevPlant p, const float* __restrict__ q, int64_t n,
                                                 float* __restrict__ tf_out) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* tf = smem + warp * per_warp_floats(p);
  float* qbuf = warp_qbuf(p, tf);
  const int64_t nbatch = (n + 31) / 32;
  for (int64_t b = (int64_t)blockIdx.x * wpb + warp; b < nbatch; b += (int64_t)gridDim.x * wpb) {
    const int64_t i = b * 32 + lane;
    if (i < n) {
      for (int k = 0; k < p.dim; ++k) qbuf[k * kRow + lane] = q[i * p.dim + k];
      fk_lane(p, qbuf, tf, lane);
      for (int l = 0; l < p.num_links; ++l) {
        int s = __ldg(p.link_slot + l);
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
          float Rs[9], ts[3];
          const float* src = tf + s * 12 * kRow + lane;
          for (int k = 0; k < 9; ++k) Rs[k] = src[k * kRow];
          for (int k = 0; k < 3; ++k) ts[k] = src[(9 + k) * kRow];
          compose(Rs, ts, Rf, tfx, R, t);
        }
        float4* dst = reinterpret_cast<float4*>(tf_out + (i * p.num_links + l) * 16);
        float last = s == -2 ? 0.f : 1.f;
        dst[0] = make_float4(R[0], R[1], R[2], 0.f);
        dst[1] = make_float4(R[3], R[4], R[5], 0.f);
        dst[2] = make_float4(R[6], R[7], R[8], 0.f);
        dst[3] = make_float4(t[0], t[1], t[2], last);
      }
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
csd_status_t launch_check_points(const csd_plant_s* p, const float* q, int64_t n, const VoxelTables& vt,
                                 uint8_t* out, cudaStream_t st) {
  if (n <= 0) return CSD_OK;
  const int wpb = 4;
  size_t smem = smem_bytes(p, wpb);
  int grid = 0;
  csd_status_t s = grid_for(check_points_kernel, smem, (n + 31) / 32, &grid, wpb);
  if (s) return s;
  VoxArgs va{vt.vox, vt.nv, vt.vr, vt.tile_mask, vt.other, vt.num_other};
  check_points_kernel<<<grid, 32 * wpb, smem, st>>>(p->dp, q, n, va, out);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_fk(const csd_plant_s* p, const float* q, int64_t n, float* tf, cudaStream_t st) {
  if (n <= 0) return CSD_OK;
  const int wpb = 4;
  size_t smem = smem_bytes(p, wpb);
  int grid = 0;
  csd_status_t s = grid_for(fk_kernel, smem, (n + 31) / 32, &grid, wpb);
  if (s) return s;
  fk_kernel<<<grid, 32 * wpb, smem, st>>>(p->dp, q, n, tf);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_check_edges(const csd_plant_s* p, const float* s0, const float* e0, int64_t n, float step,
                                int mode, uint8_t* out, int64_t* pts, unsigned int* counter, cudaStream_t st) {
  if (n <= 0) return CSD_OK;
  const int wpb = 4;
  size_t smem = smem_bytes(p, wpb);
  int grid = 0;
  csd_status_t s = grid_for(check_edges_kernel, smem, n, &grid, wpb);
  if (s) return s;
  CSD_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
  check_edges_kernel<<<grid, 32 * wpb, smem, st>>>(p->dp, s0, e0, n, step, mode, out, pts,
                                                   reinterpret_cast<unsigned long long*>(counter));
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

csd_status_t launch_pair(int ta, const float* g_dev, int tb, uint8_t* out, cudaStream_t st) {
  pair_kernel<<<1, 1, 0, st>>>(ta, g_dev, tb, out);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

}  // namespace csd
