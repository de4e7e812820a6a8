// capi.cu -- C ABI entry points for collision checks, FK and sampling
// (declared in include/csd_capi.h).
#include <cmath>
#include <cstring>
#include <vector>

#include "check_core.cuh"

namespace csd {
csd_status_t launch_pair(int ta, const float* g_dev, int tb, uint8_t* out, cudaStream_t st);

csd_status_t build_voxel_tables(csd_plant_s* p, const int32_t* ids, int nr, std::vector<uint32_t>* tab,
                                int* num_other) {
  const int T = p->dp.num_tiles;
  tab->assign(T, 0u);
  std::vector<uint32_t> other;
  for (int k = 0; k < nr; ++k) {
    int g = ids[k];
    CSD_CHECK(g >= 0 && g < (int)p->host.moving_of_geom.size(), CSD_ERR_INVALID,
              "Invalid robot geometry ID, check the SceneInspector for valid ids.");
    int m = p->host.moving_of_geom[g];
    if (m >= 0 && m < p->dp.num_msph) {
      (*tab)[m / kWarp] |= 1u << (m % kWarp);
    } else if (m >= 0) {
      other.push_back((uint32_t)m);
    } else {
      other.push_back(0x80000000u | (uint32_t)p->host.static_of_geom[g]);
    }
  }
  tab->insert(tab->end(), other.begin(), other.end());
  *num_other = (int)other.size();
  return CSD_OK;
}

// Reads and clears the plant's status word once the stream's work is done:
// nonzero when a block's bounded wait for the static-table staging gave up,
// in which case that block returned without checking its configurations.
csd_status_t plant_status(const csd_plant_s* p, cudaStream_t st) {
  int v = 0;
  CSD_CUDA_TRY(cudaMemcpyAsync(&v, p->dp.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  if (v) {
    CSD_CUDA_TRY(cudaMemsetAsync(p->dp.status, 0, sizeof(int), st));
    CSD_CUDA_TRY(cudaStreamSynchronize(st));
    set_error("a check kernel's bounded wait for the static-table staging gave up; the call's results are incomplete");
    return CSD_ERR_CUDA;
  }
  return CSD_OK;
}

namespace {

struct DeviceGuard {  // run a call on the plant's device
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = 0;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace csd

using namespace csd;

extern "C" {

uint32_t csd_num_samples_unadaptive(float epsilon, float delta, float tau) {
  float one_over = 1.0f / delta;
  float lg = std::log(one_over);
  float num = 2.0f * lg;
  float den = epsilon * tau * tau;
  return (uint32_t)std::ceil(num / den);
}

csd_status_t csd_fk(csd_plant_t p, const float* q, int64_t n, float* tf, int32_t flags, void* stream) {
  CSD_CHECK(p && n >= 0 && (n == 0 || (q && tf)), CSD_ERR_INVALID, "null argument");
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int d = p->dp.dim, L = p->dp.num_links;
  if (flags == CSD_PTR_DEVICE) return launch_fk(p, q, n, tf, st);
  csd_status_t s;
  if ((s = p->in_buf.reserve((size_t)n * d * sizeof(float) + 16))) return s;
  if ((s = p->out_buf.reserve((size_t)n * L * 16 * sizeof(float)))) return s;
  if (n * d) CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf.ptr, q, (size_t)n * d * sizeof(float), cudaMemcpyHostToDevice, st));
  if ((s = launch_fk(p, p->in_buf.as<float>(), n, p->out_buf.as<float>(), st))) return s;
  CSD_CUDA_TRY(cudaMemcpyAsync(tf, p->out_buf.ptr, (size_t)n * L * 16 * sizeof(float), cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  return CSD_OK;
}

csd_status_t csd_check_points(csd_plant_t p, const float* q, int64_t n, const float* voxels, int32_t nv, float vr,
                              const int32_t* robot_ids, int32_t nr, uint8_t* out, int32_t flags, void* stream) {
  CSD_CHECK(p && n >= 0 && (n == 0 || (q && out)), CSD_ERR_INVALID, "null argument");
  CSD_CHECK(nv >= 0 && (nv == 0 || voxels), CSD_ERR_INVALID, "null voxels");
  CSD_CHECK(nr >= 0 && (nr == 0 || robot_ids), CSD_ERR_INVALID, "null robot geometry ids");
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int d = p->dp.dim;
  VoxelTables vt;
  csd_status_t s;
  if (nv > 0 && nr > 0) {
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, robot_ids) == cudaSuccess && pa.type == cudaMemoryTypeDevice) {
      set_error("robot_geometry_ids must be host memory (they are read on the host)");
      return CSD_ERR_INVALID;
    }
    cudaGetLastError();  // an unregistered host pointer is not an error here
    std::vector<uint32_t> tab;
    int no = 0;
    if ((s = build_voxel_tables(p, robot_ids, nr, &tab, &no))) return s;
    if ((s = p->vox_tab.reserve(tab.size() * sizeof(uint32_t)))) return s;
    CSD_CUDA_TRY(cudaMemcpyAsync(p->vox_tab.ptr, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    const float* vdev = voxels;
    if (flags != CSD_PTR_DEVICE) {
      if ((s = p->vox_buf.reserve((size_t)nv * 3 * sizeof(float)))) return s;
      CSD_CUDA_TRY(cudaMemcpyAsync(p->vox_buf.ptr, voxels, (size_t)nv * 3 * sizeof(float), cudaMemcpyHostToDevice, st));
      vdev = p->vox_buf.as<float>();
    }
    vt.vox = vdev;
    vt.nv = nv;
    vt.vr = vr;
    vt.tile_mask = p->vox_tab.as<uint32_t>();
    vt.other = p->vox_tab.as<uint32_t>() + p->dp.num_tiles;
    vt.num_other = no;
    if ((s = build_voxel_grid(p, voxel_grid_cell(p, tab, vr), &p->vox_grid_buf, &vt, st))) return s;
  }
  if (flags == CSD_PTR_DEVICE) {
    s = launch_check_points(p, q, n, vt, out, st);
    if (s) return s;
    if (nv > 0 && nr > 0) return plant_status(p, st);  // synchronises: voxel tables are reused per call
    return CSD_OK;
  }
  if ((s = p->in_buf.reserve((size_t)n * d * sizeof(float) + 16))) return s;
  if ((s = p->out_buf.reserve((size_t)n + 16))) return s;
  if (n * d) CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf.ptr, q, (size_t)n * d * sizeof(float), cudaMemcpyHostToDevice, st));
  if ((s = launch_check_points(p, p->in_buf.as<float>(), n, vt, p->out_buf.as<uint8_t>(), st))) return s;
  if (n) CSD_CUDA_TRY(cudaMemcpyAsync(out, p->out_buf.ptr, (size_t)n, cudaMemcpyDeviceToHost, st));
  return plant_status(p, st);
}

csd_status_t csd_plant_status(csd_plant_t p, int32_t* timed_out, void* stream) {
  CSD_CHECK(p && timed_out, CSD_ERR_INVALID, "null argument");
  DeviceGuard g(p->device);
  const csd_status_t s = plant_status(p, (cudaStream_t)stream);
  *timed_out = s == CSD_ERR_CUDA ? 1 : 0;
  return s == CSD_ERR_CUDA ? CSD_OK : s;
}

csd_status_t csd_plant_wait_selftest(csd_plant_t p, int32_t polls, int32_t* reported) {
  CSD_CHECK(p && reported && polls >= 1, CSD_ERR_INVALID, "bad arguments");
  DeviceGuard g(p->device);
  *reported = 0;
  staging_wait_selftest_kernel<<<1, 128, 0, 0>>>(p->dp.status, (long long)polls);
  CSD_CUDA_TRY(cudaGetLastError());
  const csd_status_t s = plant_status(p, 0);
  if (s == CSD_ERR_CUDA) {
    *reported = 1;
    return CSD_OK;
  }
  return s;
}

csd_status_t csd_check_edges(csd_plant_t p, const float* starts, const float* ends, int64_t n, float step, int32_t mode,
                             uint8_t* out, int64_t* pts, int32_t flags, void* stream) {
  CSD_CHECK(p && n >= 0 && (n == 0 || (starts && ends && out)), CSD_ERR_INVALID, "null argument");
  CSD_CHECK(mode >= CSD_EDGE_L2_REF && mode <= CSD_EDGE_VG, CSD_ERR_INVALID, "bad edge discretisation mode");
  CSD_CHECK(step > 0.f && std::isfinite(step), CSD_ERR_INVALID, "step size must be positive");
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int d = p->dp.dim;
  csd_status_t s;
  if ((s = p->counter.reserve(64))) return s;
  if (flags == CSD_PTR_DEVICE)
    return launch_check_edges(p, starts, ends, n, step, mode, out, pts, p->counter.as<unsigned int>(), st);
  const size_t qb = (size_t)n * d * sizeof(float);
  if ((s = p->in_buf.reserve(qb + 16))) return s;
  if ((s = p->in_buf2.reserve(qb + 16))) return s;
  if ((s = p->out_buf.reserve((size_t)n + 16))) return s;
  if ((s = p->out_buf2.reserve((size_t)n * sizeof(int64_t) + 16))) return s;
  if (qb) {
    CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf.ptr, starts, qb, cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf2.ptr, ends, qb, cudaMemcpyHostToDevice, st));
  }
  if ((s = launch_check_edges(p, p->in_buf.as<float>(), p->in_buf2.as<float>(), n, step, mode, p->out_buf.as<uint8_t>(),
                              pts ? p->out_buf2.as<int64_t>() : nullptr, p->counter.as<unsigned int>(), st)))
    return s;
  if (n) {
    CSD_CUDA_TRY(cudaMemcpyAsync(out, p->out_buf.ptr, (size_t)n, cudaMemcpyDeviceToHost, st));
    if (pts) CSD_CUDA_TRY(cudaMemcpyAsync(pts, p->out_buf2.ptr, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  }
  return plant_status(p, st);
}

csd_status_t csd_check_edges_ranked(csd_plant_t p, csd_mlp_t mlp, int32_t net, const float* starts, const float* ends,
                                    int64_t n, float step, int32_t mode, int32_t top, uint8_t* out, int64_t* pts,
                                    int32_t flags, void* stream) {
  CSD_CHECK(p && mlp && n >= 0 && (n == 0 || (starts && ends && out)), CSD_ERR_INVALID, "null argument");
  CSD_CHECK(mode >= CSD_EDGE_L2_REF && mode <= CSD_EDGE_VG, CSD_ERR_INVALID, "bad edge discretisation mode");
  CSD_CHECK(step > 0.f && std::isfinite(step), CSD_ERR_INVALID, "step size must be positive");
  CSD_CHECK(top >= 0 && top <= 32, CSD_ERR_INVALID, "top must be in [0, 32]");
  const MlpView mv = mlp_view(mlp);
  const int d = p->dp.dim;
  CSD_CHECK(net >= 0 && net < mv.nets, CSD_ERR_INVALID, "bad net index");
  CSD_CHECK(mv.dims[net] == d, CSD_ERR_DIMENSION, "the net's input dimension differs from the plant's");
  CSD_CHECK(mv.device == p->device, CSD_ERR_INVALID, "the surrogate and the plant live on different devices");
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  csd_status_t s;
  if (n == 0) return CSD_OK;
  if ((s = p->counter.reserve(64))) return s;
  const float* sd = starts;
  const float* ed = ends;
  uint8_t* od = out;
  int64_t* pd = pts;
  const size_t qb = (size_t)n * d * sizeof(float);
  if (flags != CSD_PTR_DEVICE) {
    if ((s = p->in_buf.reserve(qb + 16)) || (s = p->in_buf2.reserve(qb + 16)) || (s = p->out_buf.reserve((size_t)n + 16)) ||
        (s = p->out_buf2.reserve((size_t)n * sizeof(int64_t) + 16)))
      return s;
    CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf.ptr, starts, qb, cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf2.ptr, ends, qb, cudaMemcpyHostToDevice, st));
    sd = p->in_buf.as<float>();
    ed = p->in_buf2.as<float>();
    od = p->out_buf.as<uint8_t>();
    pd = pts ? p->out_buf2.as<int64_t>() : nullptr;
  }
  // points per edge, their offsets, and chunks of at most kChunk scored points
  constexpr int64_t kChunk = int64_t(1) << 22;
  DevBuf cnt, offd, xb, lg;
  if ((s = cnt.reserve((size_t)n * 8 + 16)) || (s = offd.reserve((size_t)(n + 1) * 8 + 16))) return s;
  if ((s = launch_edge_count(sd, ed, n, d, step, (int)mode, cnt.as<int64_t>(), st))) return s;
  std::vector<int64_t> off(n + 1, 0);
  CSD_CUDA_TRY(cudaMemcpyAsync(off.data() + 1, cnt.ptr, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  for (int64_t i = 0; i < n; ++i) off[i + 1] += off[i];
  CSD_CUDA_TRY(cudaMemcpyAsync(offd.ptr, off.data(), (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, st));
  const int64_t most = std::min<int64_t>(off[n], kChunk);
  if (top > 0 && most > 0) {
    if ((s = xb.reserve((size_t)most * d * 4 + 16)) || (s = lg.reserve((size_t)most * 4 + 16))) return s;
  }
  for (int64_t c0 = 0; c0 < n;) {
    int64_t c1 = c0 + 1;
    while (c1 < n && off[c1 + 1] - off[c0] <= kChunk) ++c1;
    const int64_t P = off[c1] - off[c0];
    const bool ranked = top > 0 && P <= kChunk;  // an edge longer than a chunk is checked unranked
    if (ranked) {
      if ((s = launch_edge_materialize(sd, ed, c0, c1, offd.as<int64_t>(), d, (int)mode, xb.as<float>(), st))) return s;
      const int32_t rows = (int32_t)P;
      if ((s = csd_mlp_infer(mlp, 1, &net, &rows, xb.as<float>(), lg.as<float>(), CSD_PTR_DEVICE, st))) return s;
    }
    if ((s = launch_check_edges_ranked(p, sd, ed, c0, c1, offd.as<int64_t>(), ranked ? lg.as<float>() : nullptr, top,
                                       (int)mode, od, pd, p->counter.as<unsigned int>(), st)))
      return s;
    c0 = c1;
  }
  if (flags != CSD_PTR_DEVICE) {
    CSD_CUDA_TRY(cudaMemcpyAsync(out, od, (size_t)n, cudaMemcpyDeviceToHost, st));
    if (pts) CSD_CUDA_TRY(cudaMemcpyAsync(pts, pd, (size_t)n * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  }
  return plant_status(p, st);
}

csd_status_t csd_visibility_graph(csd_plant_t p, const float* nodes, int32_t n, float step, uint8_t* adjacency,
                                  int32_t flags, void* stream) {
  CSD_CHECK(p && n >= 2 && nodes && adjacency, CSD_ERR_INVALID, "a visibility graph needs at least two nodes");
  CSD_CHECK(step >= 1e-12f && std::isfinite(step), CSD_ERR_INVALID, "step size must be positive");
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int d = p->dp.dim;
  const int64_t E = (int64_t)n * (n - 1) / 2;
  csd_status_t s;
  if ((s = p->counter.reserve(64))) return s;
  if (flags == CSD_PTR_DEVICE)
    return launch_check_edges(p, nodes, nodes, E, step, CSD_EDGE_VG, adjacency, nullptr, p->counter.as<unsigned int>(),
                              st, n);
  const size_t qb = (size_t)n * d * sizeof(float);
  if ((s = p->in_buf.reserve(qb + 16)) || (s = p->out_buf.reserve((size_t)E + 16))) return s;
  CSD_CUDA_TRY(cudaMemcpyAsync(p->in_buf.ptr, nodes, qb, cudaMemcpyHostToDevice, st));
  if ((s = launch_check_edges(p, p->in_buf.as<float>(), p->in_buf.as<float>(), E, step, CSD_EDGE_VG,
                              p->out_buf.as<uint8_t>(), nullptr, p->counter.as<unsigned int>(), st, n)))
    return s;
  CSD_CUDA_TRY(cudaMemcpyAsync(adjacency, p->out_buf.ptr, (size_t)E, cudaMemcpyDeviceToHost, st));
  return plant_status(p, st);
}

csd_status_t csd_pair_collision_free(int32_t ta, const float* da, const float* XLBa, const float* XWLa, int32_t tb,
                                     const float* db, const float* XLBb, const float* XWLb, uint8_t* out) {
  CSD_CHECK(da && XLBa && XWLa && db && XLBb && XWLb && out, CSD_ERR_INVALID, "null argument");
  if (ta == G_CYLINDER || tb == G_CYLINDER) {
    set_error("Cylinders and capsules are not supported yet.");
    return CSD_ERR_UNSUPPORTED;
  }
  CSD_CHECK(ta >= 0 && ta <= G_CAPSULE && tb >= 0 && tb <= G_CAPSULE, CSD_ERR_INVALID, "bad geometry type");
  // world poses X_W_L * X_L_B in FP32 (collision_checker.cpp:96-97), then the world format
  float g[32];
  const float* XL[2] = {XLBa, XLBb};
  const float* XW[2] = {XWLa, XWLb};
  const float* dm[2] = {da, db};
  const int ty[2] = {ta, tb};
  for (int k = 0; k < 2; ++k) {
    float R[9], t[3];
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) {
        float s = 0.f;
        for (int j = 0; j < 3; ++j) s += XW[k][j * 4 + r] * XL[k][c * 4 + j];
        R[c * 3 + r] = s;
      }
    for (int r = 0; r < 3; ++r) {
      float s = XW[k][12 + r];
      for (int j = 0; j < 3; ++j) s += XW[k][j * 4 + r] * XL[k][12 + j];
      t[r] = s;
    }
    float* o = g + 16 * k;
    for (int i = 0; i < 16; ++i) o[i] = 0.f;
    if (ty[k] == G_SPHERE) {
      o[0] = t[0]; o[1] = t[1]; o[2] = t[2]; o[3] = dm[k][0];
    } else if (ty[k] == G_CAPSULE) {
      o[0] = t[0]; o[1] = t[1]; o[2] = t[2]; o[3] = dm[k][0];
      o[4] = R[6]; o[5] = R[7]; o[6] = R[8]; o[7] = 0.5f * dm[k][1];
    } else {
      for (int a = 0; a < 3; ++a) {
        o[4 * a] = R[a * 3]; o[4 * a + 1] = R[a * 3 + 1]; o[4 * a + 2] = R[a * 3 + 2];
        o[4 * a + 3] = -(R[a * 3] * t[0] + R[a * 3 + 1] * t[1] + R[a * 3 + 2] * t[2]);
        o[12 + a] = 0.5f * dm[k][a];
      }
    }
  }
  float* gd = nullptr;
  CSD_CUDA_TRY(cudaMalloc(&gd, sizeof(g) + 16));
  csd_status_t s = CSD_OK;
  if (cudaMemcpy(gd, g, sizeof(g), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("cudaMemcpy failed");
    s = CSD_ERR_CUDA;
  }
  if (!s) s = launch_pair(ta, gd, tb, reinterpret_cast<uint8_t*>(gd + 32), 0);
  if (!s && cudaMemcpy(out, gd + 32, 1, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("cudaMemcpy failed");
    s = CSD_ERR_CUDA;
  }
  cudaFree(gd);
  return s;
}

csd_status_t csd_uniform_sample_hpolyhedra(const float* A, const float* b, const int32_t* face_off, int32_t P,
                                           int32_t dim, const float* starts, int32_t S, int32_t mixing,
                                           uint64_t seed, float* samples, int32_t* num_failed, int32_t flags,
                                           void* stream) {
  CSD_CHECK(P >= 0 && S >= 0 && mixing >= 0, CSD_ERR_INVALID, "negative size");
  CSD_CHECK(dim >= 1 && dim <= kMaxDim, CSD_ERR_DIMENSION, "dimension must be in [1, 16]");
  if (P == 0 || S == 0) {
    if (num_failed) *num_failed = 0;
    return CSD_OK;
  }
  CSD_CHECK(A && b && face_off && starts && samples, CSD_ERR_INVALID, "null argument");
  cudaStream_t st = (cudaStream_t)stream;
  if (flags == CSD_PTR_DEVICE) {
    int* nf = nullptr;
    if (num_failed) {
      CSD_CUDA_TRY(cudaMallocAsync((void**)&nf, sizeof(int), st));
      CSD_CUDA_TRY(cudaMemsetAsync(nf, 0, sizeof(int), st));
    }
    csd_status_t s = launch_hit_and_run(A, b, face_off, P, dim, starts, S, mixing, seed, 0u, 0, samples, nf, nullptr, st);
    if (num_failed) {
      if (!s) {
        cudaMemcpyAsync(num_failed, nf, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
      }
      cudaFreeAsync(nf, st);
    }
    return s;
  }
  // host arrays: containment check (hpolyhedron.cpp:265-274, tolerance 1e-9)
  const int F = face_off[P];
  for (int p = 0; p < P; ++p) {
    CSD_CHECK(face_off[p] >= 0 && face_off[p] <= face_off[p + 1], CSD_ERR_INVALID, "bad face offsets");
    for (int f = face_off[p]; f < face_off[p + 1]; ++f) {
      float ax = 0.f;
      for (int k = 0; k < dim; ++k) ax += A[(int64_t)f * dim + k] * starts[(int64_t)p * dim + k];
      if (!(ax <= b[f] + 1e-9f)) {
        set_error("starting point " + std::to_string(p) + " is not contained in polytope " + std::to_string(p) +
                  ". The initial point must lie inside of the polytope.");
        return CSD_ERR_NOT_CONTAINED;
      }
    }
  }
  size_t bA = (size_t)F * dim * sizeof(float), bb = (size_t)F * sizeof(float), bo = (size_t)(P + 1) * sizeof(int32_t),
         bs = (size_t)P * dim * sizeof(float), bout = (size_t)P * S * dim * sizeof(float);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t total = al(bA) + al(bb) + al(bo) + al(bs) + al(bout) + 256;
  char* dev = nullptr;
  CSD_CUDA_TRY(cudaMalloc((void**)&dev, total));
  char* pA = dev;
  char* pb = pA + al(bA);
  char* po = pb + al(bb);
  char* ps = po + al(bo);
  char* pout = ps + al(bs);
  int* pnf = reinterpret_cast<int*>(pout + al(bout));
  csd_status_t s = CSD_OK;
  auto h2d = [&](void* dst, const void* src, size_t n) {
    if (!s && n && cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      set_error("cudaMemcpyAsync failed");
      s = CSD_ERR_CUDA;
    }
  };
  h2d(pA, A, bA);
  h2d(pb, b, bb);
  h2d(po, face_off, bo);
  h2d(ps, starts, bs);
  if (!s && cudaMemsetAsync(pnf, 0, sizeof(int), st) != cudaSuccess) s = CSD_ERR_CUDA;
  if (!s)
    s = launch_hit_and_run((const float*)pA, (const float*)pb, (const int32_t*)po, P, dim, (const float*)ps, S, mixing,
                           seed, 0u, 0, (float*)pout, pnf, nullptr, st);
  int nf = 0;
  if (!s && (cudaMemcpyAsync(samples, pout, bout, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaMemcpyAsync(&nf, pnf, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaStreamSynchronize(st) != cudaSuccess)) {
    set_error("copy back failed");
    s = CSD_ERR_CUDA;
  }
  cudaFree(dev);
  if (num_failed) *num_failed = nf;
  return s;
}

}  // extern "C"
