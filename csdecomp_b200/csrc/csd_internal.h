// csd_internal.h -- host-side handle types, error plumbing and device buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/csd_capi.h"
#include "csd_device.cuh"

namespace csd {

void set_error(const std::string& msg);

struct Status {
  csd_status_t code;
  std::string msg;
};

#define CSD_CUDA_TRY(expr)                                                               \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      ::csd::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));              \
      return CSD_ERR_CUDA;                                                               \
    }                                                                                    \
  } while (0)

#define CSD_CHECK(cond, code, msg)   \
  do {                               \
    if (!(cond)) {                   \
      ::csd::set_error(msg);         \
      return (code);                 \
    }                                \
  } while (0)

// Grow-only device buffer (no allocation once warm).
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  csd_status_t reserve(size_t n);
  ~DevBuf();
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
};

struct HostPlant {  // host copies kept for host-side checks and voxel tables
  int dim = 0;
  int num_links = 0;
  std::vector<int> moving_of_geom;  // geometry -> moving index or -1
  std::vector<int> static_of_geom;  // geometry -> static index or -1
  std::vector<int> geom_type;
  std::vector<MovingGeom> moving;
  std::vector<float> statics;       // [S][16]
  std::vector<int> static_type;
  int num_tile_pairs = 0;
  // algorithmic FP32 work of one configuration checked without early exit
  // (FMA = 2 FLOP, add/mul/min/max/compare = 1; sqrt, div and sincos not counted)
  double flops_fk = 0, flops_place = 0, flops_pairs = 0;
};

// FLOP of one evaluation of each pair test, from the code in csd_device.cuh.
constexpr double kFlopSphSph = 11, kFlopSphBox = 32, kFlopSphABox = 16, kFlopSphCap = 24, kFlopCapCap = 58, kFlopCapBox = 240,
                 kFlopBoxBox = 800;
constexpr double kFlopFkRevolute = 99, kFlopFkPrismatic = 69, kFlopFkRootRevolute = 36, kFlopFkRootPrismatic = 6;
constexpr double kFlopPlaceSphere = 18, kFlopPlaceCapsule = 33, kFlopPlaceBox = 78;
inline double pair_flops(int ta, int tb) {
  if (ta > tb) { int t = ta; ta = tb; tb = t; }
  // types: 0 box, 1 sphere, 3 capsule
  if (ta == 1 && tb == 1) return kFlopSphSph;
  if (ta == 0 && tb == 1) return kFlopSphBox;
  if (ta == 1 && tb == 3) return kFlopSphCap;
  if (ta == 3 && tb == 3) return kFlopCapCap;
  if (ta == 0 && tb == 3) return kFlopCapBox;
  return kFlopBoxBox;
}

}  // namespace csd

struct csd_plant_s {
  int device = 0;
  csd::DevPlant dp{};
  csd::HostPlant host;
  void* blob = nullptr;  // device tables
  bool cull_eligible = false;  // <= 32 slots and <= 1024 statics
  bool vox_grid = true;        // voxel checks through the hash grid (csd_plant_set_voxel_grid)
  // scratch for host-pointer calls and per-call voxel tables
  csd::DevBuf in_buf, in_buf2, out_buf, out_buf2, vox_buf, vox_tab, vox_grid_buf, counter;
  ~csd_plant_s();
};

namespace csd {

// Per-call voxel tables derived from robot geometry ids.
struct VoxelTables {
  const float* vox = nullptr;     // [V][3] device
  int nv = 0;
  float vr = 0.f;
  const uint32_t* tile_mask = nullptr;  // [num_tiles] lanes of each sphere tile checked against voxels
  const uint32_t* other = nullptr;      // geometry refs (bit31 = static) checked lane-over-voxels
  int num_other = 0;
  // hash grid over the voxels (voxgrid.cu); gstart == nullptr: no grid
  const float4* gvox = nullptr;
  const int* gstart = nullptr;
  int gmask = 0;
  float ginv_h = 0.f;
};

csd_status_t build_voxel_tables(csd_plant_s* p, const int32_t* robot_ids, int nr, std::vector<uint32_t>* tab,
                                int* num_other);
// Synchronises st, then reads and clears the plant's status word (capi.cu):
// CSD_ERR_CUDA when a block's bounded staging wait gave up since the last read.
csd_status_t plant_status(const csd_plant_s* p, cudaStream_t st);
// Cell edge of the voxel grid for these tables (tab from build_voxel_tables):
// twice the median radius of the robot spheres checked against voxels plus
// the voxel radius.
float voxel_grid_cell(const csd_plant_s* p, const std::vector<uint32_t>& tab, float vr);
// Builds the hash grid of the device voxels vt->vox (vt->nv of them) into buf
// on stream st and fills vt's grid fields, when the plant's grid switch is on
// and there are at least kVoxGridMinVoxels voxels; otherwise leaves them null.
csd_status_t build_voxel_grid(const csd_plant_s* p, float cell, DevBuf* buf, VoxelTables* vt, cudaStream_t st);

// kernels (check.cu)
csd_status_t launch_check_points(const csd_plant_s* p, const float* q, int64_t n, const VoxelTables& vt,
                                 uint8_t* out, cudaStream_t st);
csd_status_t launch_fk(const csd_plant_s* p, const float* q, int64_t n, float* tf, cudaStream_t st);
csd_status_t launch_check_edges(const csd_plant_s* p, const float* s, const float* e, int64_t n, float step,
                                int mode, uint8_t* out, int64_t* pts, unsigned int* counter, cudaStream_t st, int64_t nodes = 0);
// surrogate-ranked edge checks (check.cu)
csd_status_t launch_edge_count(const float* s, const float* e, int64_t n, int d, float step, int mode,
                               int64_t* counts, cudaStream_t st);
csd_status_t launch_edge_materialize(const float* s, const float* e, int64_t e0, int64_t e1, const int64_t* off, int d,
                                     int mode, float* x, cudaStream_t st);
csd_status_t launch_check_edges_ranked(const csd_plant_s* p, const float* s0, const float* e0p, int64_t e0, int64_t e1,
                                       const int64_t* off, const float* logits, int top, int mode, uint8_t* out,
                                       int64_t* pts, unsigned int* counter, cudaStream_t st);
// sampler.cu
csd_status_t launch_hit_and_run(const float* A, const float* b, const int32_t* face_off, int num_poly, int dim,
                                const float* starts, int samples_per_poly, int mixing, uint64_t seed,
                                uint32_t stream_base, int fail_keep, float* out, int* num_failed,
                                const int* num_faces_dev, cudaStream_t st);
// EI-ZO sampler over one region stored as face-pair rows (sampler_core.cuh,
// pair_stride(dim) floats per row, start slacks at `start`); the face count is
// read on the device. A failed chain keeps its start point.
csd_status_t launch_sample_region(const float* rows, const int* num_faces_dev, int dim, const float* start, int S,
                                  int mixing, uint64_t seed, uint32_t stream, float* out, cudaStream_t st);
// Face-pair rows of faces [0, F) of row-major A and b (start slacks at x0).
csd_status_t launch_put_faces(const float* A, const float* b, int F, int dim, const float* x0, float* rows,
                              cudaStream_t st);

int device_sm_count();

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`, never lowering it: handles and calls with different plants
// launch the same kernels with different shared-memory sizes, and a lower
// limit set by one (another handle, another thread) would make the others'
// launches fail.
template <typename K>
inline cudaError_t raise_smem_limit(K kernel, size_t bytes) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kernel));
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)bytes);
}

// The surrogate bank's device tensors (mlp.cu): bf16 weights, f32 parameters,
// input scale, and the input dimension of each net.
struct MlpView {
  const void* wb;
  const float* params;
  float in_scale;
  int nets;
  const int* dims;  // host array
  int device;
};
MlpView mlp_view(csd_mlp_t h);

}  // namespace csd
