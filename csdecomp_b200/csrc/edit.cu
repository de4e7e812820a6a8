// edit.cu -- region editing (EditRegionsCuda) on the device.
//
// Reference: EditRegionsCuda (csdecomp/src/planning/cuda_edit_regions.cu:44-301)
// groups the collisions by segment on the host, then launches a projection
// kernel and 9 x (midpoint, FK, voxel check, bounds, store) plus a distance
// kernel, each step through global-memory transform and per-pair buffers, and
// places the faces on the host: per region an argsort of the distances and an
// Eigen loop that tests every candidate against all faces so far.
//
// Here the editing is two launches after one upload:
//   1. edit_bisect_kernel   one warp per collision: projection onto its own
//                            segment, every bisection step a fused FK + pair
//                            check of the midpoint with the link-level broad
//                            phase, distance to the projection (the EI-ZO
//                            bisection body, bisect_particle)
//   2. edit_faces_kernel    one warp per region: copies the region, drops the
//                            candidates outside it, then repeatedly takes the
//                            nearest live candidate (lower index on ties),
//                            places its face with the segment relaxation of
//                            cuda_edit_regions.cu:262-272 and drops every
//                            candidate the new face cuts off. A candidate is
//                            placed exactly when the reference's ascending
//                            loop finds it strictly inside the region edited
//                            so far (:253-259): faces only accumulate, so
//                            "inside all faces so far" is "not cut off by the
//                            original region nor by a face placed before it".
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>

#include "eizo_core.cuh"

namespace csd {

constexpr int kEditFaceThreads = 256;
constexpr int kEditMaxVoxels = 10000;  // MAX_NUM_VOXELS, cuda_edge_inflation_zero_order.h:13

template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3)
    edit_bisect_kernel(DevPlant p, int K, int dim, int steps, const float* __restrict__ starts,
                       const float* __restrict__ ends, const uint32_t* __restrict__ seg, VoxArgs va,
                       float* __restrict__ cols, float* __restrict__ proj, float* __restrict__ dist) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  const WarpCtx<SM> w = warp_setup<SM>(p, smem4, &bar);
  if (!w.ok) return;
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < K; i += nw) {
    const size_t s = (size_t)seg[i] * dim;
    bisect_particle<SM>(p, w, i, dim, steps, starts + s, ends + s, va, cols, proj, dist, lane);
  }
}

// Region r: faces [face_off[r], face_off[r+1]) of A/b, candidates
// [coll_off[r], coll_off[r+1]) of cols/proj/dist; written at row
// face_off[r] + coll_off[r] of A_out/b_out. One warp per region (shuffles and
// warp barriers only; kEditFaceThreads / 32 regions per block). dist is
// consumed (FLT_MAX marks a candidate that is placed or cut off). Lane 0
// computes each face with the coordinate-order arithmetic of the oracle.
__global__ void __launch_bounds__(kEditFaceThreads)
    edit_faces_kernel(int m, int dim, float margin, const float* __restrict__ starts, const float* __restrict__ ends,
                      const float* __restrict__ A, const float* __restrict__ b, const int* __restrict__ face_off,
                      const int* __restrict__ coll_off, const float* __restrict__ cols,
                      const float* __restrict__ proj, float* __restrict__ dist, float* __restrict__ A_out,
                      float* __restrict__ b_out, int* __restrict__ num_faces) {
  __shared__ float face_s[kEditFaceThreads / 32][kMaxDim + 1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float* face = face_s[wib];
  const int nwarps = gridDim.x * (kEditFaceThreads / 32);
  for (int r = blockIdx.x * (kEditFaceThreads / 32) + wib; r < m; r += nwarps) {
    const int f0 = face_off[r], F0 = face_off[r + 1] - f0;
    const int c0 = coll_off[r], K = coll_off[r + 1] - c0;
    const int64_t row0 = (int64_t)f0 + c0;
    float* Ao = A_out + row0 * dim;
    float* bo = b_out + row0;
    const float* Ar = A + (int64_t)f0 * dim;
    const float* br = b + f0;
    for (int i = lane; i < F0 * dim; i += 32) Ao[i] = Ar[i];
    for (int i = lane; i < F0; i += 32) bo[i] = br[i];
    const float* cr = cols + (int64_t)c0 * dim;
    const float* pr = proj + (int64_t)c0 * dim;
    float* dr = dist + c0;
    // candidates not strictly inside the original region are never placed
    for (int i = lane; i < K; i += 32) {
      const float* x = cr + (int64_t)i * dim;
      bool inside = dr[i] < FLT_MAX;
      for (int f = 0; f < F0 && inside; ++f) {
        float v = 0.f;
        for (int k = 0; k < dim; ++k) v = __fmaf_rn(Ar[(int64_t)f * dim + k], x[k], v);
        if (!(__fsub_rn(v, br[f]) < 0.f)) inside = false;
      }
      if (!inside) dr[i] = FLT_MAX;
    }
    __syncwarp();
    const float* ls = starts + (int64_t)r * dim;
    const float* le = ends + (int64_t)r * dim;
    int nf = F0;
    for (;;) {
      // nearest live candidate, lower index on ties
      float bv = FLT_MAX;
      int bi = 0x7fffffff;
      for (int i = lane; i < K; i += 32) {
        const float v = dr[i];
        if (v < bv) {  // ascending i: the first of equal values is kept
          bv = v;
          bi = i;
        }
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov < bv || (ov == bv && oi < bi)) {
          bv = ov;
          bi = oi;
        }
      }
      if (!(bv < FLT_MAX)) break;
      if (lane == 0) {
        const int sidx = bi;
        const float* c = cr + (int64_t)sidx * dim;
        const float* q = pr + (int64_t)sidx * dim;
        float a[kMaxDim];
        float n2 = 0.f;
        for (int k = 0; k < dim; ++k) {
          a[k] = __fsub_rn(c[k], q[k]);
          n2 = __fmaf_rn(a[k], a[k], n2);
        }
        if (n2 > 0.f) {  // a zero normal stays zero (Eigen's normalize)
          const float nrm = __fsqrt_rn(n2);
          for (int k = 0; k < dim; ++k) a[k] = __fdiv_rn(a[k], nrm);
        }
        float bb = 0.f, v1 = 0.f, v2 = 0.f;
        for (int k = 0; k < dim; ++k) {
          bb = __fmaf_rn(a[k], c[k], bb);
          v1 = __fmaf_rn(a[k], ls[k], v1);
          v2 = __fmaf_rn(a[k], le[k], v2);
        }
        bb = __fsub_rn(bb, margin);
        v1 = __fsub_rn(v1, bb);
        v2 = __fsub_rn(v2, bb);
        const float relax = v2 > v1 ? v2 : v1;
        // b_face += relaxation + 2e-6, evaluated in double as in the reference
        if (relax > 0.f) bb = __double2float_rn(__dadd_rn((double)bb, __dadd_rn((double)relax, 2e-6)));
        for (int k = 0; k < dim; ++k) {
          Ao[(int64_t)nf * dim + k] = a[k];
          face[k] = a[k];
        }
        bo[nf] = bb;
        face[dim] = bb;
        dr[sidx] = FLT_MAX;
      }
      __syncwarp();
      const float bb = face[dim];
      for (int i = lane; i < K; i += 32) {
        if (!(dr[i] < FLT_MAX)) continue;
        const float* x = cr + (int64_t)i * dim;
        float v = 0.f;
        for (int k = 0; k < dim; ++k) v = __fmaf_rn(face[k], x[k], v);
        if (!(__fsub_rn(v, bb) < 0.f)) dr[i] = FLT_MAX;
      }
      ++nf;
      __syncwarp();
    }
    if (lane == 0) num_faces[r] = nf;
    __syncwarp();
  }
}

static bool point_in_region(const float* A, const float* b, int F, int d, const float* x) {
  // HPolyhedron::PointInSet (hpolyhedron.cpp:265-274), tolerance 1e-9 in FP32
  for (int f = 0; f < F; ++f) {
    float ax = 0.f;
    for (int k = 0; k < d; ++k) ax += A[(size_t)f * d + k] * x[k];
    if (!(ax <= b[f] + 1e-9f)) return false;
  }
  return true;
}

}  // namespace csd

using namespace csd;

extern "C" {

csd_status_t csd_edit_regions(csd_plant_t plant, const float* collisions, const uint32_t* line_segment_idxs,
                              int64_t n, const float* line_starts, const float* line_ends, int32_t m,
                              const float* A, const float* b, const int32_t* face_offsets, const float* voxels,
                              int32_t nv, float voxel_radius, const int32_t* robot_geometry_ids, int32_t nr,
                              const csd_edit_regions_options_t* options, float* A_out, float* b_out,
                              int32_t* num_faces, float* projections, float* optimized_collisions) {
  CSD_CHECK(plant && options && line_starts && line_ends && face_offsets && A && b && A_out && b_out && num_faces,
            CSD_ERR_INVALID, "null argument");
  CSD_CHECK(m >= 1, CSD_ERR_INVALID, "Regions vector cannot be empty");
  CSD_CHECK(n >= 0 && nv >= 0 && nr >= 0, CSD_ERR_INVALID, "negative size");
  // cuda_edit_regions.cu:55-83
  CSD_CHECK(nr >= 1 && robot_geometry_ids, CSD_ERR_INVALID, "Robot geometry IDs cannot be empty");
  CSD_CHECK(voxel_radius > 0.f, CSD_ERR_INVALID, "Voxel radius must be positive");
  CSD_CHECK(nv <= kEditMaxVoxels, CSD_ERR_CAPACITY, "Voxel buffer size insufficient");
  CSD_CHECK(nv == 0 || voxels, CSD_ERR_INVALID, "null voxels");
  const int d = plant->dp.dim;
  CSD_CHECK(d >= 1 && d <= kMaxDim, CSD_ERR_DIMENSION, "plant dimension must be in [1, 16]");
  CSD_CHECK(face_offsets[0] == 0, CSD_ERR_INVALID, "face_offsets[0] must be 0");
  for (int r = 0; r < m; ++r) {
    const int F = face_offsets[r + 1] - face_offsets[r];
    CSD_CHECK(F >= 0, CSD_ERR_INVALID, "face offsets must not decrease");
    const float* Ar = A + (size_t)face_offsets[r] * d;
    const float* br = b + face_offsets[r];
    CSD_CHECK(point_in_region(Ar, br, F, d, line_starts + (size_t)r * d), CSD_ERR_NOT_CONTAINED,
              "line start is not contained in region " + std::to_string(r));
    CSD_CHECK(point_in_region(Ar, br, F, d, line_ends + (size_t)r * d), CSD_ERR_NOT_CONTAINED,
              "line end is not contained in region " + std::to_string(r));
  }
  CSD_CHECK(n >= 1, CSD_ERR_INVALID,
            "[EditRegionsCuda] No collisions are contained in the regions, this is not supported.");
  CSD_CHECK(collisions && line_segment_idxs && projections && optimized_collisions, CSD_ERR_INVALID,
            "null argument");
  CSD_CHECK(n <= 0x7fffffff, CSD_ERR_CAPACITY, "too many collisions");
  // stable grouping by segment (cuda_edit_regions.cu:85-107)
  std::vector<int> coff(m + 1, 0);
  for (int64_t i = 0; i < n; ++i) {
    CSD_CHECK(line_segment_idxs[i] < (uint32_t)m, CSD_ERR_INVALID, "line segment index out of range");
    ++coff[line_segment_idxs[i] + 1];
  }
  for (int r = 0; r < m; ++r) coff[r + 1] += coff[r];
  const int F_total = face_offsets[m];
  std::vector<int> fill(coff.begin(), coff.end() - 1);
  std::vector<float> grouped((size_t)n * d);
  std::vector<uint32_t> gseg(n);
  for (int64_t i = 0; i < n; ++i) {
    const uint32_t s = line_segment_idxs[i];
    const int j = fill[s]++;
    std::memcpy(&grouped[(size_t)j * d], collisions + (size_t)i * d, sizeof(float) * d);
    gseg[j] = s;
  }
  std::vector<uint32_t> vtab;
  int num_other = 0;
  csd_status_t s;
  if ((s = build_voxel_tables(plant, robot_geometry_ids, nr, &vtab, &num_other))) return s;

  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != plant->device) cudaSetDevice(plant->device);
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, plant->device};

  // one device allocation for the call
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t sz_cols = al((size_t)n * d * 4), sz_dist = al((size_t)n * 4), sz_seg = al((size_t)n * 4);
  const size_t sz_ends = al((size_t)m * d * 4), sz_A = al((size_t)std::max(F_total, 1) * d * 4);
  const size_t sz_b = al((size_t)std::max(F_total, 1) * 4), sz_off = al((size_t)(m + 1) * 4);
  const size_t cap = (size_t)F_total + n;
  const size_t sz_Ao = al(cap * d * 4), sz_bo = al(cap * 4), sz_nf = al((size_t)m * 4);
  const size_t sz_vox = al((size_t)std::max(nv, 1) * 12), sz_vt = al((vtab.size() + 1) * 4);
  const size_t total = 2 * sz_cols + sz_dist + sz_seg + 2 * sz_ends + sz_A + sz_b + 2 * sz_off + sz_Ao + sz_bo +
                       sz_nf + sz_vox + sz_vt;
  DevBuf buf, grid_buf;
  if ((s = buf.reserve(total))) return s;
  char* base = buf.as<char>();
  size_t off = 0;
  auto take = [&](size_t x) {
    char* p = base + off;
    off += x;
    return p;
  };
  float* cols = (float*)take(sz_cols);
  float* proj = (float*)take(sz_cols);
  float* dist = (float*)take(sz_dist);
  uint32_t* seg = (uint32_t*)take(sz_seg);
  float* ls = (float*)take(sz_ends);
  float* le = (float*)take(sz_ends);
  float* Ad = (float*)take(sz_A);
  float* bd = (float*)take(sz_b);
  int* foff = (int*)take(sz_off);
  int* coffd = (int*)take(sz_off);
  float* Ao = (float*)take(sz_Ao);
  float* bo = (float*)take(sz_bo);
  int* nfd = (int*)take(sz_nf);
  float* vox = (float*)take(sz_vox);
  uint32_t* vt = (uint32_t*)take(sz_vt);
  const cudaStream_t st = 0;
  CSD_CUDA_TRY(cudaMemcpyAsync(cols, grouped.data(), (size_t)n * d * 4, cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(seg, gseg.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(ls, line_starts, (size_t)m * d * 4, cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(le, line_ends, (size_t)m * d * 4, cudaMemcpyHostToDevice, st));
  if (F_total) {
    CSD_CUDA_TRY(cudaMemcpyAsync(Ad, A, (size_t)F_total * d * 4, cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(bd, b, (size_t)F_total * 4, cudaMemcpyHostToDevice, st));
  }
  CSD_CUDA_TRY(cudaMemcpyAsync(foff, face_offsets, (size_t)(m + 1) * 4, cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(coffd, coff.data(), (size_t)(m + 1) * 4, cudaMemcpyHostToDevice, st));
  if (nv) CSD_CUDA_TRY(cudaMemcpyAsync(vox, voxels, (size_t)nv * 12, cudaMemcpyHostToDevice, st));
  if (!vtab.empty()) CSD_CUDA_TRY(cudaMemcpyAsync(vt, vtab.data(), vtab.size() * 4, cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemsetAsync(plant->dp.status, 0, 4, st));
  VoxelTables vtab_dev;
  if (nv > 0) {
    vtab_dev.vox = vox;
    vtab_dev.nv = nv;
    vtab_dev.vr = voxel_radius;
    vtab_dev.tile_mask = vt;
    vtab_dev.other = vt + plant->dp.num_tiles;
    vtab_dev.num_other = num_other;
    if ((s = build_voxel_grid(plant, voxel_grid_cell(plant, vtab, voxel_radius), &grid_buf, &vtab_dev, st)))
      return s;
  }
  const VoxArgs va = vox_args(vtab_dev);

  // 1. bisection, one warp per collision
  const int K = (int)n, steps = (int)options->bisection_steps;
  const bool sm = statics_in_smem(plant);
  const size_t smem = smem_bytes(plant, kWarpsPerBlock);
  int grid = 0;
  if (sm) {
    if ((s = grid_for(edit_bisect_kernel<true>, smem, K, &grid, kWarpsPerBlock))) return s;
    edit_bisect_kernel<true><<<grid, 32 * kWarpsPerBlock, smem, st>>>(plant->dp, K, d, steps, ls, le, seg, va, cols,
                                                                      proj, dist);
  } else {
    if ((s = grid_for(edit_bisect_kernel<false>, smem, K, &grid, kWarpsPerBlock))) return s;
    edit_bisect_kernel<false><<<grid, 32 * kWarpsPerBlock, smem, st>>>(plant->dp, K, d, steps, ls, le, seg, va,
                                                                       cols, proj, dist);
  }
  CSD_CUDA_TRY(cudaGetLastError());
  // 2. faces, one warp per region
  const int fgrid = std::min((m + kEditFaceThreads / 32 - 1) / (kEditFaceThreads / 32), 8 * device_sm_count());
  edit_faces_kernel<<<fgrid, kEditFaceThreads, 0, st>>>(m, d, options->configuration_margin, ls, le, Ad, bd, foff,
                                                        coffd, cols, proj, dist, Ao, bo, nfd);
  CSD_CUDA_TRY(cudaGetLastError());
  int kstat = 0;
  CSD_CUDA_TRY(cudaMemcpyAsync(num_faces, nfd, (size_t)m * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(&kstat, plant->dp.status, 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(A_out, Ao, cap * d * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(b_out, bo, cap * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(projections, proj, (size_t)n * d * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(optimized_collisions, cols, (size_t)n * d * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  CSD_CHECK(kstat == 0, CSD_ERR_CUDA, "static geometry staging timed out in the bisection kernel");
  return CSD_OK;
}

}  // extern "C"
