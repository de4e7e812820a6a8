// eizo.cu -- EI-ZO edge inflation on the device.
//
// Reference: executeEizo (csdecomp/src/planning/cuda_edge_inflation_zero_order.cu:94-339)
// drives each iteration from the host with ~12 + 3*faces launches and
// blocking copies: sample, FK, pair check, pool, atomicAdd compaction (D2H),
// first-M count (D2H), projection, 9 x (midpoint, FK, check, pool, bounds,
// store), distances, then per face a thrust::min_element, a <<<1,1>>>
// maybePlaceFace with two memcpys and a redundancy kernel.
//
// Here an iteration is five launches and one 16-byte device-to-host read:
//   1. sample_region_kernel         M_k chains in the current region (face-pair
//                                    rows, slacks carried from step to step)
//   2. check_points_kernel          fused FK + pair sweep, one verdict byte each
//   3. compact_kernel               one block: ordered prefix scan of the
//                                    colliding samples (the reference's atomicAdd
//                                    slot order is scheduling dependent,
//                                    cuda_set_builder_utils.cu:168-186) and the
//                                    first-M collision count
//   -- host reads the counts, applies the admissibility test --
//   4. bisect_kernel                projection onto the segment and all
//                                    bisection steps, each step a fused FK +
//                                    check of the 32 midpoints a warp owns
//   5. faces_kernel                 one block: greedy argmin (first index on
//                                    ties, as thrust::min_element), face
//                                    placement with the segment relaxation
//                                    (cuda_set_builder_utils.cu:359-401) and
//                                    redundancy marking (:402-424), all faces
//                                    of the iteration in one launch.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "eizo_core.cuh"

namespace csd {

__global__ void compact_kernel(const uint8_t* __restrict__ flags, const float* __restrict__ samples, int N, int M,
                               int max_keep, int dim, float* __restrict__ cols, EizoCounters* cnt) {
  compact_block(flags, samples, N, M, max_keep, dim, cols, cnt);
}

template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) bisect_kernel(DevPlant p, int K, int dim, int steps,
                                                                       const float* __restrict__ ls,
                                                                       const float* __restrict__ le, VoxArgs va,
                                                                       float* __restrict__ cols,
                                                                       float* __restrict__ proj,
                                                                       float* __restrict__ dist) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  const WarpCtx<SM> w = warp_setup<SM>(p, smem4, &bar);
  if (!w.ok) return;
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < K; i += nw)
    bisect_particle<SM>(p, w, i, dim, steps, ls, le, va, cols, proj, dist, lane);
}

// One block places up to max_faces faces (greedy, nearest collision first).
__global__ void __launch_bounds__(1024) faces_kernel(int K, int dim, int max_faces, int capacity, float margin,
                                                     const float* __restrict__ ls, const float* __restrict__ le,
                                                     const float* __restrict__ cols, const float* __restrict__ proj,
                                                     float* __restrict__ dist, float* __restrict__ A,
                                                     float* __restrict__ b, int* __restrict__ num_faces,
                                                     EizoCounters* cnt, float* __restrict__ rows) {
  faces_block(K, dim, max_faces, capacity, margin, ls, le, cols, proj, dist, A, b, num_faces, cnt, rows);
}

}  // namespace csd

// ------------------------------------------------------------------- handle
struct csd_inflator_s {
  csd_plant_s* plant = nullptr;
  int device = 0;
  int dim = 0;
  csd_eizo_options_t opt{};
  int domain_faces = 0;
  int capacity = 0;
  int max_voxels = 0;
  int max_configs = 0;
  std::vector<float> domain_A, domain_b;
  std::vector<uint32_t> vtab_host;
  int num_other = 0;
  csd::DevBuf A, rows, b, nf, samples, flags, cols, proj, dist, seg, vox, vtab, vgrid, cnt;
  csd::EizoCounters* host_cnt = nullptr;  // pinned
  int* host_nf = nullptr;                 // pinned
  // last inflate, track_iteration_information and dim <= 3: the collision points after
  // bisection of each iteration that placed faces ([K][dim] each), for plotting
  std::vector<std::vector<float>> points_post_bisection;
  ~csd_inflator_s() {
    if (host_cnt) cudaFreeHost(host_cnt);
    if (host_nf) cudaFreeHost(host_nf);
  }
};

namespace csd {

static bool point_in_set(const std::vector<float>& A, const std::vector<float>& b, int F, int d, const float* x) {
  for (int f = 0; f < F; ++f) {
    float ax = 0.f;
    for (int k = 0; k < d; ++k) ax += A[(size_t)f * d + k] * x[k];
    if (!(ax <= b[f] + 1e-9f)) return false;
  }
  return true;
}

static csd_status_t launch_bisect(const csd_plant_s* p, int K, int dim, int steps, const float* ls, const float* le,
                                  const VoxArgs& va, float* cols, float* proj, float* dist, cudaStream_t st) {
  if (K <= 0) return CSD_OK;
  const bool sm = statics_in_smem(p);
  const size_t smem = (size_t)warp_floats(p->dp) * sizeof(float) * kWarpsPerBlock + (sm ? p->dp.static_bytes : 0);
  int grid = 0;
  csd_status_t s;
  if (sm) {
    if ((s = grid_for(bisect_kernel<true>, smem, K, &grid, kWarpsPerBlock))) return s;
    bisect_kernel<true><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, K, dim, steps, ls, le, va, cols, proj, dist);
  } else {
    if ((s = grid_for(bisect_kernel<false>, smem, K, &grid, kWarpsPerBlock))) return s;
    bisect_kernel<false><<<grid, 32 * kWarpsPerBlock, smem, st>>>(p->dp, K, dim, steps, ls, le, va, cols, proj, dist);
  }
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

}  // namespace csd

using namespace csd;

extern "C" {

csd_status_t csd_inflator_create(csd_plant_t plant, const int32_t* ids, int32_t nr, const csd_eizo_options_t* o,
                                 const float* dA, const float* db, int32_t F0, int32_t max_voxels, int32_t capacity,
                                 csd_inflator_t* out) {
  CSD_CHECK(plant && o && out && (F0 == 0 || (dA && db)) && (nr == 0 || ids), CSD_ERR_INVALID, "null argument");
  CSD_CHECK(F0 >= 0 && nr >= 0 && max_voxels >= 0, CSD_ERR_INVALID, "negative size");
  *out = nullptr;
  const int d = plant->dp.dim;
  CSD_CHECK(d >= 1 && d <= kMaxDim, CSD_ERR_DIMENSION, "plant dimension must be in [1, 16]");
  CSD_CHECK(capacity >= F0 && capacity > 0, CSD_ERR_CAPACITY, "face capacity smaller than the domain");
  CSD_CHECK(capacity <= kMaxRegionFaces, CSD_ERR_CAPACITY, "face capacity above 4096 (the sampler's largest region)");
  CSD_CHECK(o->num_particles >= 1 && o->max_iterations >= 1, CSD_ERR_INVALID, "num_particles and max_iterations must be positive");
  CSD_CHECK(o->tau > 0.f && o->tau < 1.f && o->epsilon > 0.f && o->delta > 0.f, CSD_ERR_INVALID, "bad epsilon/delta/tau");
  // EizoGpuMemory sizing, cuda_edge_inflation_zero_order.cu:448-494
  double delta_min = 6 * o->delta / (M_PI * M_PI * (double)o->max_iterations * (double)o->max_iterations);
  uint32_t mmax = csd_num_samples_unadaptive(o->epsilon, (float)delta_min, o->tau);
  if (o->num_particles > mmax) {
    set_error("Current required particle count exceeds buffer size. There were " + std::to_string(o->num_particles) +
              " num_particles requested, and " + std::to_string(mmax) +
              " max_num_configurations space provided by the unadaptive test.");
    return CSD_ERR_CAPACITY;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != plant->device) cudaSetDevice(plant->device);
  std::unique_ptr<csd_inflator_s> h(new csd_inflator_s());
  h->plant = plant;
  h->device = plant->device;
  h->dim = d;
  h->opt = *o;
  h->domain_faces = F0;
  h->capacity = capacity;
  h->max_voxels = max_voxels;
  h->max_configs = (int)std::max<uint32_t>(mmax, o->num_particles);
  h->domain_A.assign(dA, dA + (size_t)F0 * d);
  h->domain_b.assign(db, db + F0);
  csd_status_t s;
  if ((s = build_voxel_tables(plant, ids, nr, &h->vtab_host, &h->num_other))) return s;
  const size_t np = o->num_particles, mc = (size_t)h->max_configs;
  if ((s = h->A.reserve((size_t)capacity * d * 4)) ||
      (s = h->rows.reserve(((size_t)capacity / 2 + 1) * pair_stride(d) * 4)) ||
      (s = h->b.reserve((size_t)capacity * 4)) ||
      (s = h->nf.reserve(16)) || (s = h->samples.reserve(mc * d * 4)) || (s = h->flags.reserve(mc + 16)) ||
      (s = h->cols.reserve(np * d * 4)) || (s = h->proj.reserve(np * d * 4)) || (s = h->dist.reserve(np * 4)) ||
      (s = h->seg.reserve(2 * d * 4)) || (s = h->vox.reserve((size_t)std::max(1, max_voxels) * 12)) ||
      (s = h->vtab.reserve((h->vtab_host.size() + 1) * 4)) || (s = h->cnt.reserve(sizeof(EizoCounters))))
    return s;
  if (F0) {
    CSD_CUDA_TRY(cudaMemcpy(h->A.ptr, dA, (size_t)F0 * d * 4, cudaMemcpyHostToDevice));
    CSD_CUDA_TRY(cudaMemcpy(h->b.ptr, db, (size_t)F0 * 4, cudaMemcpyHostToDevice));
  }
  if (!h->vtab_host.empty())
    CSD_CUDA_TRY(cudaMemcpy(h->vtab.ptr, h->vtab_host.data(), h->vtab_host.size() * 4, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaMallocHost((void**)&h->host_cnt, sizeof(EizoCounters)));
  CSD_CUDA_TRY(cudaMallocHost((void**)&h->host_nf, sizeof(int) * 4));
  if (cur != plant->device) cudaSetDevice(cur);
  *out = h.release();
  return CSD_OK;
}

csd_status_t csd_inflator_destroy(csd_inflator_t h) {
  if (!h) return CSD_OK;
  int cur = 0, dev = h->device;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  delete h;
  if (cur != dev) cudaSetDevice(cur);
  return CSD_OK;
}

csd_status_t csd_inflator_inflate(csd_inflator_t h, const float* ls, const float* le, const float* voxels, int32_t nv,
                                  float vr, float* A_out, float* b_out, int32_t* num_faces,
                                  csd_eizo_iteration_info_t* info, int32_t info_cap, int32_t* num_iters, void* stream) {
  CSD_CHECK(h && ls && le && A_out && b_out && num_faces, CSD_ERR_INVALID, "null argument");
  CSD_CHECK(nv >= 0 && (nv == 0 || voxels), CSD_ERR_INVALID, "null voxels");
  CSD_CHECK(nv <= h->max_voxels, CSD_ERR_CAPACITY, "more voxels than the inflator was created for");
  const int d = h->dim;
  CSD_CHECK(point_in_set(h->domain_A, h->domain_b, h->domain_faces, d, ls) &&
                point_in_set(h->domain_A, h->domain_b, h->domain_faces, d, le),
            CSD_ERR_NOT_CONTAINED, "line segment endpoints must lie in the domain");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, h->device};
  cudaStream_t st = (cudaStream_t)stream;
  const csd_eizo_options_t& o = h->opt;
  csd_plant_s* p = h->plant;
  // reset the region to the domain and upload the segment and voxels
  h->host_nf[0] = h->domain_faces;
  CSD_CUDA_TRY(cudaMemcpyAsync(h->nf.ptr, h->host_nf, sizeof(int), cudaMemcpyHostToDevice, st));
  std::vector<float> seg(2 * d);
  std::memcpy(seg.data(), ls, d * 4);
  std::memcpy(seg.data() + d, le, d * 4);
  CSD_CUDA_TRY(cudaMemcpyAsync(h->seg.ptr, seg.data(), 2 * d * 4, cudaMemcpyHostToDevice, st));
  if (nv) CSD_CUDA_TRY(cudaMemcpyAsync(h->vox.ptr, voxels, (size_t)nv * 12, cudaMemcpyHostToDevice, st));
  const float* ls_d = h->seg.as<float>();
  const float* le_d = ls_d + d;
  csd_status_t s;
  // the domain's face-pair rows with their slacks at this segment's start
  if ((s = launch_put_faces(h->A.as<float>(), h->b.as<float>(), h->domain_faces, d, ls_d, h->rows.as<float>(), st)))
    return s;
  VoxelTables vt;
  if (nv > 0 && !h->vtab_host.empty()) {
    vt.vox = h->vox.as<float>();
    vt.nv = nv;
    vt.vr = vr;
    vt.tile_mask = h->vtab.as<uint32_t>();
    vt.other = h->vtab.as<uint32_t>() + p->dp.num_tiles;
    vt.num_other = h->num_other;
    if ((s = build_voxel_grid(p, voxel_grid_cell(p, h->vtab_host, vr), &h->vgrid, &vt, st))) return s;
  }
  const VoxArgs va = vox_args(vt);
  EizoCounters* cnt = h->cnt.as<EizoCounters>();
  const bool keep_points = o.track_iteration_information && d <= 3;
  h->points_post_bisection.clear();
  int nit = 0;
  int last_with_faces = -1;
  auto t_prev = std::chrono::high_resolution_clock::now();
  for (uint32_t it = 0; it < o.max_iterations; ++it) {
    auto t0 = std::chrono::high_resolution_clock::now();
    float delta_k = (float)(6 * o.delta / (M_PI * M_PI * (it + 1) * (it + 1)));
    uint32_t M = csd_num_samples_unadaptive(o.epsilon, delta_k, o.tau);
    uint32_t N = std::max(M, o.num_particles);
    if ((s = launch_sample_region(h->rows.as<float>(), h->nf.as<int>(), d, ls_d, (int)N, (int)o.mixing_steps, o.seed,
                                  0u, h->samples.as<float>(), st)))
      return s;
    if ((s = launch_check_points(p, h->samples.as<float>(), N, vt, h->flags.as<uint8_t>(), st))) return s;
    compact_kernel<<<1, 1024, 0, st>>>(h->flags.as<uint8_t>(), h->samples.as<float>(), (int)N, (int)M,
                                       (int)o.num_particles, d, h->cols.as<float>(), cnt);
    CSD_CUDA_TRY(cudaGetLastError());
    CSD_CUDA_TRY(cudaMemcpyAsync(h->host_cnt, cnt, sizeof(EizoCounters), cudaMemcpyDeviceToHost, st));
    CSD_CUDA_TRY(cudaStreamSynchronize(st));
    if (last_with_faces >= 0) {
      if (info && last_with_faces < info_cap) info[last_with_faces].num_faces_placed = (int32_t)h->host_cnt->placed;
      if (h->host_cnt->status == 2) {
        set_error("Max face count exceeded.");
        return CSD_ERR_CAPACITY;
      }
      last_with_faces = -1;
    }
    const uint32_t total = h->host_cnt->total, first_m = h->host_cnt->first_m;
    const float thr = (1 - o.tau) * o.epsilon * M;
    csd_eizo_iteration_info_t rec{};
    rec.iteration_index = (int32_t)it;
    rec.num_samples_drawn = (int32_t)N;
    rec.collisions_threshold = (int32_t)thr;
    rec.num_collisions_unadaptive = (int32_t)first_m;
    if (o.verbose)
      printf("iter %u, num collisions found in first M samples %u, thresh %f\n", it, first_m, (double)thr);
    if ((float)first_m <= thr) {
      auto t1 = std::chrono::high_resolution_clock::now();
      rec.iteration_time_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
      if (info && nit < info_cap) info[nit] = rec;
      ++nit;
      break;
    }
    const uint32_t K = std::min(total, o.num_particles);
    if ((s = launch_bisect(p, (int)K, d, (int)o.bisection_steps, ls_d, le_d, va, h->cols.as<float>(),
                           h->proj.as<float>(), h->dist.as<float>(), st)))
      return s;
    if (keep_points) {  // as executeEizo keeps them for dim <= 3 (cuda_edge_inflation_zero_order.cu:323-335)
      h->points_post_bisection.resize(nit + 1);
      std::vector<float>& pts = h->points_post_bisection[nit];
      pts.resize((size_t)K * d);
      CSD_CUDA_TRY(cudaMemcpyAsync(pts.data(), h->cols.ptr, pts.size() * 4, cudaMemcpyDeviceToHost, st));
    }
    faces_kernel<<<1, 1024, 0, st>>>((int)K, d, (int)o.max_hyperplanes_per_iteration, h->capacity,
                                     o.configuration_margin, ls_d, le_d, h->cols.as<float>(), h->proj.as<float>(),
                                     h->dist.as<float>(), h->A.as<float>(), h->b.as<float>(), h->nf.as<int>(), cnt,
                                     h->rows.as<float>());
    CSD_CUDA_TRY(cudaGetLastError());
    rec.num_collisions_updated = (int32_t)K;
    auto t1 = std::chrono::high_resolution_clock::now();
    rec.iteration_time_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
    if (info && nit < info_cap) info[nit] = rec;
    last_with_faces = nit;
    ++nit;
    (void)t_prev;
  }
  CSD_CUDA_TRY(cudaMemcpyAsync(h->host_cnt, cnt, sizeof(EizoCounters), cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(h->host_nf, h->nf.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  if (last_with_faces >= 0) {
    if (info && last_with_faces < info_cap) info[last_with_faces].num_faces_placed = (int32_t)h->host_cnt->placed;
    if (h->host_cnt->status == 2) {
      set_error("Max face count exceeded.");
      return CSD_ERR_CAPACITY;
    }
  }
  const int F = h->host_nf[0];
  CSD_CUDA_TRY(cudaMemcpyAsync(A_out, h->A.ptr, (size_t)F * d * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(b_out, h->b.ptr, (size_t)F * 4, cudaMemcpyDeviceToHost, st));
  if ((s = plant_status(p, st))) return s;
  *num_faces = F;
  if (num_iters) *num_iters = nit;
  return CSD_OK;
}

csd_status_t csd_inflator_points_post_bisection(csd_inflator_t h, int32_t iteration, float* points, int32_t capacity,
                                               int32_t* count) {
  CSD_CHECK(h && count && iteration >= 0 && (capacity == 0 || points), CSD_ERR_INVALID, "bad arguments");
  *count = 0;
  if (iteration >= (int32_t)h->points_post_bisection.size()) return CSD_OK;
  const std::vector<float>& pts = h->points_post_bisection[iteration];
  *count = (int32_t)(pts.size() / h->dim);
  const size_t n = std::min<size_t>(pts.size(), (size_t)capacity * h->dim);
  if (n) std::memcpy(points, pts.data(), n * 4);
  return CSD_OK;
}

csd_status_t csd_eizo(csd_plant_t plant, const float* ls, const float* le, const float* voxels, int32_t nv, float vr,
                      const float* dA, const float* db, int32_t F0, const int32_t* ids, int32_t nr,
                      const csd_eizo_options_t* o, int32_t capacity, float* A_out, float* b_out, int32_t* num_faces,
                      csd_eizo_iteration_info_t* info, int32_t info_cap, int32_t* num_iters) {
  CSD_CHECK(plant && o, CSD_ERR_INVALID, "null argument");
  // EizoCuda argument checks, cuda_edge_inflation_zero_order.cu:355-386
  CSD_CHECK(F0 <= 0.9 * capacity, CSD_ERR_CAPACITY,
            "The domain polyhedron is already reserving almost all of the allocated faces.");
  csd_inflator_t h = nullptr;
  csd_status_t s = csd_inflator_create(plant, ids, nr, o, dA, db, F0, nv, capacity, &h);
  if (s) return s;
  s = csd_inflator_inflate(h, ls, le, voxels, nv, vr, A_out, b_out, num_faces, info, info_cap, num_iters, nullptr);
  csd_inflator_destroy(h);
  return s;
}

}  // extern "C"

// ---------------------------------------------------------- allocation-free EI-ZO
// csd_eizo_noalloc: the one-shot inflation for callers that must not allocate
// device memory during the call. Its scratch (samples, verdict bytes,
// collision points, projections, distances, the region being grown, segment,
// voxel tables, counters) is carved from one file-scope device array; the
// plant handle is created beforehand. Host code cannot pass the array's name
// to a kernel (in host code it is a stand-in, not a device address), so the
// first call on each device looks the address up with cudaGetSymbolAddress.
#include <mutex>

namespace csd {

constexpr size_t kNoAllocScratchBytes = size_t(2) << 20;  // 2 MiB per device, held until process exit
constexpr int kNoAllocMaxTiles = 64;
constexpr int kNoAllocMaxRobotIds = 1024;

static __device__ __align__(256) unsigned char g_eizo_scratch[kNoAllocScratchBytes];

static std::mutex g_scratch_mu;
static void* g_scratch_addr[64] = {nullptr};

// Device address of g_eizo_scratch on the current device (looked up once per device).
static csd_status_t scratch_address(int dev, unsigned char** out) {
  CSD_CHECK(dev >= 0 && dev < 64, CSD_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    CSD_CUDA_TRY(cudaGetSymbolAddress(&p, g_eizo_scratch));
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return CSD_OK;
}

}  // namespace csd

extern "C" csd_status_t csd_eizo_noalloc(csd_plant_t plant, const float* ls, const float* le, const float* voxels,
                                         int32_t nv, float vr, const float* dA, const float* db, int32_t F0,
                                         const int32_t* ids, int32_t nr, const csd_eizo_options_t* o,
                                         int32_t capacity, float* A_out, float* b_out, int32_t* num_faces,
                                         csd_eizo_iteration_info_t* info, int32_t info_cap, int32_t* num_iters,
                                         void* stream) {
  using namespace csd;
  CSD_CHECK(plant && o && ls && le && A_out && b_out && num_faces, CSD_ERR_INVALID, "null argument");
  CSD_CHECK(F0 >= 0 && (F0 == 0 || (dA && db)) && nr >= 0 && (nr == 0 || ids) && nv >= 0 && (nv == 0 || voxels),
            CSD_ERR_INVALID, "bad domain, robot geometry or voxel arguments");
  const int d = plant->dp.dim;
  CSD_CHECK(d >= 1 && d <= kMaxDim, CSD_ERR_DIMENSION, "plant dimension must be in [1, 16]");
  CSD_CHECK(capacity >= F0 && capacity > 0 && F0 <= 0.9 * capacity, CSD_ERR_CAPACITY,
            "The domain polyhedron is already reserving almost all of the allocated faces.");
  CSD_CHECK(capacity <= kMaxRegionFaces, CSD_ERR_CAPACITY, "face capacity above 4096 (the sampler's largest region)");
  CSD_CHECK(o->num_particles >= 1 && o->max_iterations >= 1, CSD_ERR_INVALID,
            "num_particles and max_iterations must be positive");
  CSD_CHECK(o->tau > 0.f && o->tau < 1.f && o->epsilon > 0.f && o->delta > 0.f, CSD_ERR_INVALID,
            "bad epsilon/delta/tau");
  double delta_min = 6 * o->delta / (M_PI * M_PI * (double)o->max_iterations * (double)o->max_iterations);
  const uint32_t mmax = csd_num_samples_unadaptive(o->epsilon, (float)delta_min, o->tau);
  CSD_CHECK(o->num_particles <= mmax, CSD_ERR_CAPACITY,
            "Current required particle count exceeds buffer size of the unadaptive test.");
  CSD_CHECK(plant->dp.num_tiles <= kNoAllocMaxTiles && nr <= kNoAllocMaxRobotIds, CSD_ERR_CAPACITY,
            "csd_eizo_noalloc supports at most 2048 moving spheres and 1024 robot geometry ids");
  // point-in-domain check of the segment (as CudaEdgeInflator::inflateEdge asserts)
  for (int s = 0; s < 2; ++s) {
    const float* x = s ? le : ls;
    for (int f = 0; f < F0; ++f) {
      float ax = 0.f;
      for (int k = 0; k < d; ++k) ax += dA[(size_t)f * d + k] * x[k];
      CSD_CHECK(ax <= db[f] + 1e-9f, CSD_ERR_NOT_CONTAINED, "line segment endpoints must lie in the domain");
    }
  }
  // ---- carve the scratch
  const size_t max_configs = std::max<uint32_t>(mmax, o->num_particles), np = o->num_particles;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t vtab_words = (size_t)plant->dp.num_tiles + (size_t)nr;
  const size_t sz_A = al((size_t)capacity * d * 4), sz_b = al((size_t)capacity * 4), sz_nf = 256,
               sz_rows = al(((size_t)capacity / 2 + 1) * pair_stride(d) * 4),
               sz_samples = al(max_configs * d * 4), sz_flags = al(max_configs), sz_cols = al(np * d * 4),
               sz_dist = al(np * 4), sz_seg = al(2 * (size_t)d * 4), sz_vox = al((size_t)nv * 12),
               sz_vtab = al(vtab_words * 4), sz_cnt = 256;
  const size_t need = sz_A + sz_rows + sz_b + sz_nf + sz_samples + sz_flags + 2 * sz_cols + sz_dist + sz_seg + sz_vox +
                      sz_vtab + sz_cnt;
  if (need > kNoAllocScratchBytes) {
    set_error("csd_eizo_noalloc needs " + std::to_string(need) + " bytes of scratch for these options, more than its " +
              std::to_string(kNoAllocScratchBytes) +
              "-byte array (fewer particles, faces, voxels or unadaptive samples fit)");
    return CSD_ERR_CAPACITY;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != plant->device) cudaSetDevice(plant->device);
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, plant->device};
  unsigned char* base = nullptr;
  csd_status_t s = scratch_address(plant->device, &base);
  if (s) return s;
  unsigned char* at = base;
  auto take = [&](size_t n) {
    unsigned char* p = at;
    at += n;
    return p;
  };
  float* A = (float*)take(sz_A);
  float* rows = (float*)take(sz_rows);
  float* b = (float*)take(sz_b);
  int* nf = (int*)take(sz_nf);
  float* samples = (float*)take(sz_samples);
  uint8_t* flags = (uint8_t*)take(sz_flags);
  float* cols = (float*)take(sz_cols);
  float* proj = (float*)take(sz_cols);
  float* dist = (float*)take(sz_dist);
  float* seg = (float*)take(sz_seg);
  float* vox = (float*)take(sz_vox);
  uint32_t* vtab = (uint32_t*)take(sz_vtab);
  EizoCounters* cnt = (EizoCounters*)take(sz_cnt);
  cudaStream_t st = (cudaStream_t)stream;
  // voxel tables from the robot geometry ids (fixed-size host arrays, no allocation)
  uint32_t vt_host[kNoAllocMaxTiles + kNoAllocMaxRobotIds];
  int num_other = 0;
  const int T = plant->dp.num_tiles;
  for (int t = 0; t < T; ++t) vt_host[t] = 0u;
  for (int k = 0; k < nr; ++k) {
    int g = ids[k];
    CSD_CHECK(g >= 0 && g < (int)plant->host.moving_of_geom.size(), CSD_ERR_INVALID, "Invalid robot geometry ID");
    int m = plant->host.moving_of_geom[g];
    if (m >= 0 && m < plant->dp.num_msph)
      vt_host[m / kWarp] |= 1u << (m % kWarp);
    else
      vt_host[T + num_other++] = m >= 0 ? (uint32_t)m : (0x80000000u | (uint32_t)plant->host.static_of_geom[g]);
  }
  // calls share the array: clear the counters, then reset region, segment and voxels
  CSD_CUDA_TRY(cudaMemsetAsync(cnt, 0, sz_cnt, st));
  if (F0) {
    CSD_CUDA_TRY(cudaMemcpyAsync(A, dA, (size_t)F0 * d * 4, cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(b, db, (size_t)F0 * 4, cudaMemcpyHostToDevice, st));
  }
  int nf_host = F0;
  CSD_CUDA_TRY(cudaMemcpyAsync(nf, &nf_host, sizeof(int), cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(seg, ls, d * 4, cudaMemcpyHostToDevice, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(seg + d, le, d * 4, cudaMemcpyHostToDevice, st));
  if (nv) CSD_CUDA_TRY(cudaMemcpyAsync(vox, voxels, (size_t)nv * 12, cudaMemcpyHostToDevice, st));
  if (vtab_words) CSD_CUDA_TRY(cudaMemcpyAsync(vtab, vt_host, (T + num_other) * 4, cudaMemcpyHostToDevice, st));
  if ((s = launch_put_faces(A, b, F0, d, seg, rows, st))) return s;  // the domain's face-pair rows
  CSD_CUDA_TRY(cudaStreamSynchronize(st));  // host staging arrays go out of scope below
  VoxelTables vt;
  if (nv > 0 && nr > 0) {
    vt.vox = vox;
    vt.nv = nv;
    vt.vr = vr;
    vt.tile_mask = vtab;
    vt.other = vtab + T;
    vt.num_other = num_other;
  }
  const VoxArgs va = vox_args(vt);
  EizoCounters hc{};
  int nit = 0, last_with_faces = -1;
  for (uint32_t it = 0; it < o->max_iterations; ++it) {
    auto t0 = std::chrono::high_resolution_clock::now();
    float delta_k = (float)(6 * o->delta / (M_PI * M_PI * (it + 1) * (it + 1)));
    uint32_t M = csd_num_samples_unadaptive(o->epsilon, delta_k, o->tau);
    uint32_t N = std::max(M, o->num_particles);
    if ((s = launch_sample_region(rows, nf, d, seg, (int)N, (int)o->mixing_steps, o->seed, 0u, samples, st)))
      return s;
    if ((s = launch_check_points(plant, samples, N, vt, flags, st))) return s;
    compact_kernel<<<1, 1024, 0, st>>>(flags, samples, (int)N, (int)M, (int)o->num_particles, d, cols, cnt);
    CSD_CUDA_TRY(cudaGetLastError());
    CSD_CUDA_TRY(cudaMemcpyAsync(&hc, cnt, sizeof(EizoCounters), cudaMemcpyDeviceToHost, st));
    CSD_CUDA_TRY(cudaStreamSynchronize(st));
    if (last_with_faces >= 0) {
      if (info && last_with_faces < info_cap) info[last_with_faces].num_faces_placed = (int32_t)hc.placed;
      if (hc.status == 2) {
        set_error("Max face count exceeded.");
        return CSD_ERR_CAPACITY;
      }
      last_with_faces = -1;
    }
    const float thr = (1 - o->tau) * o->epsilon * M;
    csd_eizo_iteration_info_t rec{};
    rec.iteration_index = (int32_t)it;
    rec.num_samples_drawn = (int32_t)N;
    rec.collisions_threshold = (int32_t)thr;
    rec.num_collisions_unadaptive = (int32_t)hc.first_m;
    if ((float)hc.first_m <= thr) {
      rec.iteration_time_ms =
          std::chrono::duration<float, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
      if (info && nit < info_cap) info[nit] = rec;
      ++nit;
      break;
    }
    const uint32_t K = std::min(hc.total, o->num_particles);
    if ((s = launch_bisect(plant, (int)K, d, (int)o->bisection_steps, seg, seg + d, va, cols, proj, dist, st))) return s;
    faces_kernel<<<1, 1024, 0, st>>>((int)K, d, (int)o->max_hyperplanes_per_iteration, capacity,
                                     o->configuration_margin, seg, seg + d, cols, proj, dist, A, b, nf, cnt,
                                     rows);
    CSD_CUDA_TRY(cudaGetLastError());
    rec.num_collisions_updated = (int32_t)K;
    rec.iteration_time_ms =
        std::chrono::duration<float, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
    if (info && nit < info_cap) info[nit] = rec;
    last_with_faces = nit;
    ++nit;
  }
  CSD_CUDA_TRY(cudaMemcpyAsync(&hc, cnt, sizeof(EizoCounters), cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(&nf_host, nf, sizeof(int), cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  if (last_with_faces >= 0) {
    if (info && last_with_faces < info_cap) info[last_with_faces].num_faces_placed = (int32_t)hc.placed;
    if (hc.status == 2) {
      set_error("Max face count exceeded.");
      return CSD_ERR_CAPACITY;
    }
  }
  CSD_CUDA_TRY(cudaMemcpyAsync(A_out, A, (size_t)nf_host * d * 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaMemcpyAsync(b_out, b, (size_t)nf_host * 4, cudaMemcpyDeviceToHost, st));
  if ((s = plant_status(plant, st))) return s;
  *num_faces = nf_host;
  if (num_iters) *num_iters = nit;
  return CSD_OK;
}
