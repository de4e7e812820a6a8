// check_core.cuh -- warp-level collision checking shared by the check and
// EI-ZO kernels (see check.cu for the design).
#pragma once
#include <algorithm>

#include "csd_internal.h"

namespace csd {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRow = 33;  // shared-memory row stride (floats) of the slot table

struct VoxArgs {
  const float* vox;
  int nv;
  float vr;
  const uint32_t* tile_mask;
  const uint32_t* other;
  int num_other;
};

// Per-warp shared memory (floats): slot table [slots][12][kRow], the batch's
// configurations [kMaxDim][kRow], moving world poses [pose_words].
static __device__ __forceinline__ int per_warp_floats(const DevPlant& p) {
  return p.num_slots * 12 * kRow + kMaxDim * kRow + ((p.pose_words + 3) & ~3);
}
static __device__ __forceinline__ float* warp_qbuf(const DevPlant& p, float* tf) { return tf + p.num_slots * 12 * kRow; }
static __device__ __forceinline__ float* warp_pose(const DevPlant& p, float* tf) {
  return tf + p.num_slots * 12 * kRow + kMaxDim * kRow;
}

static __device__ __forceinline__ void load_fk_joint(const FkJoint* src, FkJoint& J) {
  const float4* s4 = reinterpret_cast<const float4*>(src);
  float4* d4 = reinterpret_cast<float4*>(&J);
#pragma unroll
  for (int i = 0; i < 10; ++i) d4[i] = __ldg(s4 + i);
}

// FK of the configuration in column `lane` of the warp's configuration
// buffer (qbuf[k * kRow + lane]) by one lane into the slot table.
static __device__ __forceinline__ void fk_lane(const DevPlant& p, const float* qbuf, float* tf, int lane) {
  for (int j = 0; j < p.num_fk; ++j) {
    FkJoint J;
    load_fk_joint(p.fk + j, J);
    float Rl[9], tl[3], R[9], t[3];
    joint_local(J, qbuf[J.qidx * kRow + lane], Rl, tl);
    if (J.parent < 0) {
#pragma unroll
      for (int i = 0; i < 9; ++i) R[i] = Rl[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) t[i] = tl[i];
    } else {
      float Rp[9], tp[3];
      const float* src = tf + J.parent * 12 * kRow + lane;
#pragma unroll
      for (int i = 0; i < 9; ++i) Rp[i] = src[i * kRow];
#pragma unroll
      for (int i = 0; i < 3; ++i) tp[i] = src[(9 + i) * kRow];
      compose(Rp, tp, Rl, tl, R, t);
    }
    float* dst = tf + J.child * 12 * kRow + lane;
#pragma unroll
    for (int i = 0; i < 9; ++i) dst[i * kRow] = R[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) dst[(9 + i) * kRow] = t[i];
  }
}

// Moving-geometry world poses of configuration c of the batch.
static __device__ __forceinline__ void place_all(const DevPlant& p, const float* tf, float* pose, int c, int lane) {
  for (int m = lane; m < p.num_moving; m += kWarp) {
    const float4* s4 = reinterpret_cast<const float4*>(p.moving + m);
    MovingGeom g;
    float4* d4 = reinterpret_cast<float4*>(&g);
    d4[0] = __ldg(s4 + 0);
    d4[1] = __ldg(s4 + 1);
    d4[2] = __ldg(s4 + 2);
    d4[3] = __ldg(s4 + 3);
    if (g.type == G_BOX) {
      d4[4] = __ldg(s4 + 4);
      d4[5] = __ldg(s4 + 5);
      d4[6] = __ldg(s4 + 6);
    }
    float R[9], t[3];
    const float* src = tf + g.slot * 12 * kRow + c;
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = src[i * kRow];
#pragma unroll
    for (int i = 0; i < 3; ++i) t[i] = src[(9 + i) * kRow];
    float out[16];
    place_moving(g, R, t, out);
    float* dst = pose + g.pose_off;
    int nw = g.type == G_SPHERE ? 4 : g.type == G_CAPSULE ? 8 : 16;
    for (int i = 0; i < nw; i += 4) *reinterpret_cast<float4*>(dst + i) = make_float4(out[i], out[i + 1], out[i + 2], out[i + 3]);
  }
}

static __device__ __forceinline__ void load_static(const DevPlant& p, int s, int nw, float* out) {
  const float4* s4 = p.statics + 4 * s;
  for (int i = 0; i < nw / 4; ++i) {
    float4 v = __ldg(s4 + i);
    out[4 * i] = v.x;
    out[4 * i + 1] = v.y;
    out[4 * i + 2] = v.z;
    out[4 * i + 3] = v.w;
  }
}

// Geometry reference (bit 31 = static) -> type and world pose.
static __device__ __forceinline__ int load_ref(const DevPlant& p, const float* pose, uint32_t ref, float* out) {
  if (ref & 0x80000000u) {
    int s = (int)(ref & 0x7fffffffu);
    int ty = __ldg(p.static_type + s);
    load_static(p, s, ty == G_SPHERE ? 4 : ty == G_CAPSULE ? 8 : 16, out);
    return ty;
  }
  int4 h = __ldg(reinterpret_cast<const int4*>(p.moving + ref));
  int ty = h.x;
  int nw = ty == G_SPHERE ? 4 : ty == G_CAPSULE ? 8 : 16;
  const float* src = pose + h.z;
  for (int i = 0; i < nw; ++i) out[i] = src[i];
  return ty;
}

// Sphere tile t against all static geometries (dense tiles). Returns the
// warp-uniform "some pair collides".
static __device__ bool sweep_dense(const DevPlant& p, const float* pose, int t, int lane) {
  const int m = t * kWarp + lane;
  float c[4];
  if (m < p.num_msph) {
    float4 v = *reinterpret_cast<const float4*>(pose + 4 * m);
    c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
  } else {
    c[0] = c[1] = c[2] = 1e30f;
    c[3] = 0.f;
  }
  bool hit = false;
  int s = 0;
  const int s_sph = p.num_ssph, s_box = s_sph + p.num_sbox, s_end = s_box + p.num_scap;
  for (; s < s_sph; ++s) {
    float S[4];
    load_static(p, s, 4, S);
    hit |= sph_sph_hit(c, S);
    if ((s & 7) == 7 && __any_sync(kFull, hit)) return true;
  }
  if (__any_sync(kFull, hit)) return true;
  for (; s + 1 < s_box; s += 2) {
    float B0[16], B1[16];
    load_static(p, s, 16, B0);
    load_static(p, s + 1, 16, B1);
    hit |= sph_box_hit(c, c[3], B0) | sph_box_hit(c, c[3], B1);
    if ((s & 6) == 6 && __any_sync(kFull, hit)) return true;
  }
  for (; s < s_box; ++s) {
    float B[16];
    load_static(p, s, 16, B);
    hit |= sph_box_hit(c, c[3], B);
  }
  if (__any_sync(kFull, hit)) return true;
  for (; s < s_end; ++s) {
    float C[8];
    load_static(p, s, 8, C);
    hit |= sph_cap_hit(c, C);
    if ((s & 3) == 3 && __any_sync(kFull, hit)) return true;
  }
  return __any_sync(kFull, hit);
}

// Sphere tile t against the static geometries listed in its entries.
static __device__ bool sweep_masked(const DevPlant& p, const float* pose, int t, int lane) {
  const TileInfo ti = p.tiles[t];
  const int m = t * kWarp + lane;
  float c[4];
  if (m < p.num_msph) {
    float4 v = *reinterpret_cast<const float4*>(pose + 4 * m);
    c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
  } else {
    c[0] = c[1] = c[2] = 1e30f;
    c[3] = 0.f;
  }
  bool hit = false;
  int e = ti.ent_begin;
  for (; e < ti.ent_sph_end; ++e) {
    TileEntry en = p.entries[e];
    float S[4];
    load_static(p, en.s, 4, S);
    hit |= ((en.mask >> lane) & 1u) && sph_sph_hit(c, S);
    if ((e & 7) == 7 && __any_sync(kFull, hit)) return true;
  }
  for (; e < ti.ent_box_end; ++e) {
    TileEntry en = p.entries[e];
    float B[16];
    load_static(p, en.s, 16, B);
    hit |= ((en.mask >> lane) & 1u) && sph_box_hit(c, c[3], B);
    if ((e & 3) == 3 && __any_sync(kFull, hit)) return true;
  }
  for (; e < ti.ent_end; ++e) {
    TileEntry en = p.entries[e];
    float C[8];
    load_static(p, en.s, 8, C);
    hit |= ((en.mask >> lane) & 1u) && sph_cap_hit(c, C);
    if ((e & 3) == 3 && __any_sync(kFull, hit)) return true;
  }
  return __any_sync(kFull, hit);
}

static __device__ bool sweep_generic(const DevPlant& p, const float* pose, int lane) {
  for (int base = 0; base < p.num_generic; base += kWarp) {
    int k = base + lane;
    bool hit = false;
    if (k < p.num_generic) {
      GenericPair gp = p.generic[k];
      float A[16], B[16];
      int ta = load_ref(p, pose, gp.a, A);
      int tb = load_ref(p, pose, gp.b, B);
      hit = pair_hit(ta, A, tb, B);
    }
    if (__any_sync(kFull, hit)) return true;
  }
  return false;
}

static __device__ bool sweep_voxels(const DevPlant& p, const float* pose, const VoxArgs& va, int lane) {
  for (int t = 0; t < p.num_tiles; ++t) {
    uint32_t mask = va.tile_mask[t];
    if (!mask) continue;
    const int m = t * kWarp + lane;
    float c[4] = {1e30f, 1e30f, 1e30f, 0.f};
    if (m < p.num_msph) {
      float4 v = *reinterpret_cast<const float4*>(pose + 4 * m);
      c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
    }
    const bool mine = (mask >> lane) & 1u;
    bool hit = false;
    for (int v = 0; v < va.nv; ++v) {
      float S[4] = {__ldg(va.vox + 3 * v), __ldg(va.vox + 3 * v + 1), __ldg(va.vox + 3 * v + 2), va.vr};
      hit |= mine && sph_sph_hit(c, S);
      if ((v & 7) == 7 && __any_sync(kFull, hit)) return true;
    }
    if (__any_sync(kFull, hit)) return true;
  }
  for (int o = 0; o < va.num_other; ++o) {
    float G[16];
    int tg = load_ref(p, pose, va.other[o], G);
    for (int base = 0; base < va.nv; base += kWarp) {
      int v = base + lane;
      bool hit = false;
      if (v < va.nv) {
        float S[4] = {va.vox[3 * v], va.vox[3 * v + 1], va.vox[3 * v + 2], va.vr};
        hit = pair_hit(G_SPHERE, S, tg, G);
      }
      if (__any_sync(kFull, hit)) return true;
    }
  }
  return false;
}

// Full check of configuration c of the batch (warp-uniform result: true = colliding).
static __device__ bool check_config(const DevPlant& p, const float* tf, float* pose, int c, int lane, const VoxArgs& va) {
  __syncwarp();
  place_all(p, tf, pose, c, lane);
  __syncwarp();
  if (p.always_colliding) return true;
  for (int t = 0; t < p.num_tiles; ++t) {
    bool h = p.tiles[t].dense ? sweep_dense(p, pose, t, lane) : sweep_masked(p, pose, t, lane);
    if (h) return true;
  }
  if (sweep_generic(p, pose, lane)) return true;
  if (va.nv > 0 && sweep_voxels(p, pose, va, lane)) return true;
  return false;
}

// ---- host helpers shared by the launchers
static inline size_t smem_bytes(const csd_plant_s* p, int wpb) {
  size_t per = (size_t)p->dp.num_slots * 12 * kRow + (size_t)kMaxDim * kRow +
               (((size_t)p->dp.pose_words + 3) & ~size_t(3));
  return per * sizeof(float) * wpb;
}

template <typename K>
static csd_status_t grid_for(K kernel, size_t smem, int64_t work_warps, int* grid, int wpb) {
  int per_sm = 0;
  CSD_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CSD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * wpb, smem));
  if (per_sm <= 0) {
    set_error("plant tables do not fit in shared memory");
    return CSD_ERR_CAPACITY;
  }
  int64_t need = (work_warps + wpb - 1) / wpb;
  int64_t full = (int64_t)per_sm * device_sm_count();
  *grid = (int)std::max<int64_t>(1, std::min(need, full));
  return CSD_OK;
}

}  // namespace csd
