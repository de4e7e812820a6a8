// voxgrid.cu -- per-call spatial hash grid over the voxels of a voxel check.
//
// Reference: checkCollisionFreeVoxelsCuda (cuda_collision_checker.cu:374-435)
// tests every robot geometry against every voxel (a pair buffer of
// geometries x MAX_NUM_VOXELS per configuration). Here the voxels of a call
// are bucketed once on the device (count, scan, scatter: three launches,
// O(voxels)), and each robot geometry tests only the voxels in the cells its
// bounding sphere touches (check_core.cuh::grid_geom_hit). The cell edge is
// about a robot sphere's diameter plus the voxel diameter, so a sphere visits
// at most 8 cells.
#include <algorithm>
#include <vector>

#include "check_core.cuh"

namespace csd {

__global__ void vox_count_kernel(const float* __restrict__ vox, int nv, float inv_h, int mask, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const uint32_t b = vox_bucket(vox_cell(vox[3 * i], inv_h), vox_cell(vox[3 * i + 1], inv_h),
                                  vox_cell(vox[3 * i + 2], inv_h), mask);
    atomicAdd(cnt + b, 1);
  }
}

// One block: exclusive scan of the bucket counts in place (start[B] = total),
// copied to the scatter cursors.
__global__ void __launch_bounds__(1024) vox_scan_kernel(int* __restrict__ start, int* __restrict__ cursor, int B) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int per = (B + 1023) / 1024;
  const int b0 = min(t * per, B), b1 = min(b0 + per, B);
  int s = 0;
  for (int b = b0; b < b1; ++b) s += start[b];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = t ? part[t - 1] : 0;
  for (int b = b0; b < b1; ++b) {
    const int c = start[b];
    start[b] = run;
    cursor[b] = run;
    run += c;
  }
  if (t == 1023) start[B] = part[1023];
}

__global__ void vox_fill_kernel(const float* __restrict__ vox, int nv, float inv_h, int mask, int* __restrict__ cursor,
                                float4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
    const float x = vox[3 * i], y = vox[3 * i + 1], z = vox[3 * i + 2];
    const uint32_t b = vox_bucket(vox_cell(x, inv_h), vox_cell(y, inv_h), vox_cell(z, inv_h), mask);
    out[atomicAdd(cursor + b, 1)] = make_float4(x, y, z, 0.f);
  }
}

float voxel_grid_cell(const csd_plant_s* p, const std::vector<uint32_t>& tab, float vr) {
  std::vector<float> r;
  const int T = p->dp.num_tiles;
  for (int t = 0; t < T && t < (int)tab.size(); ++t)
    for (int l = 0; l < kWarp; ++l)
      if ((tab[t] >> l) & 1u) r.push_back(p->host.moving[t * kWarp + l].r);
  float med = 0.05f;
  if (!r.empty()) {
    std::nth_element(r.begin(), r.begin() + r.size() / 2, r.end());
    med = r[r.size() / 2];
  }
  return std::max(2.f * (med + std::max(vr, 0.f)), 1e-3f);
}

csd_status_t build_voxel_grid(const csd_plant_s* p, float cell, DevBuf* buf, VoxelTables* vt, cudaStream_t st) {
  vt->gvox = nullptr;
  vt->gstart = nullptr;
  if (!p->vox_grid || vt->nv < kVoxGridMinVoxels || !(cell > 0.f)) return CSD_OK;
  const int nv = vt->nv;
  int B = 256;
  while (B < 2 * nv && B < (1 << 24)) B <<= 1;
  const size_t o_cur = ((size_t)(B + 1) * 4 + 15) & ~size_t(15);
  const size_t o_vox = o_cur + (((size_t)B * 4 + 15) & ~size_t(15));
  csd_status_t s;
  if ((s = buf->reserve(o_vox + (size_t)nv * 16))) return s;
  char* base = buf->as<char>();
  int* start = reinterpret_cast<int*>(base);
  int* cursor = reinterpret_cast<int*>(base + o_cur);
  float4* gvox = reinterpret_cast<float4*>(base + o_vox);
  const float inv_h = 1.f / cell;
  CSD_CUDA_TRY(cudaMemsetAsync(start, 0, (size_t)(B + 1) * 4, st));
  const int grid = std::max(1, std::min((nv + 255) / 256, 4 * device_sm_count()));
  vox_count_kernel<<<grid, 256, 0, st>>>(vt->vox, nv, inv_h, B - 1, start);
  vox_scan_kernel<<<1, 1024, 0, st>>>(start, cursor, B);
  vox_fill_kernel<<<grid, 256, 0, st>>>(vt->vox, nv, inv_h, B - 1, cursor, gvox);
  CSD_CUDA_TRY(cudaGetLastError());
  vt->gvox = gvox;
  vt->gstart = start;
  vt->gmask = B - 1;
  vt->ginv_h = inv_h;
  return CSD_OK;
}

}  // namespace csd

using namespace csd;

extern "C" {

csd_status_t csd_plant_set_voxel_grid(csd_plant_t plant, int32_t enable) {
  CSD_CHECK(plant, CSD_ERR_INVALID, "null argument");
  plant->vox_grid = enable != 0;
  return CSD_OK;
}

}  // extern "C"
