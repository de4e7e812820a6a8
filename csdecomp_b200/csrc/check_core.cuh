// check_core.cuh -- warp-level collision checking shared by the check, edge and
// EI-ZO kernels.
//
// One warp checks one configuration:
//   1. FK, lane-parallel: lane j evaluates sin/cos of joint j, then for each
//      moving joint lanes 0..11 compute one entry of its 3x4 world transform
//      (R column-major 0..8, t 9..11) from the parent's entries in shared
//      memory and the joint's local entries exchanged by warp shuffles.
//   2. Placement, lane = moving geometry: world poses to shared memory.
//   3. Sweep: a lane holds one moving sphere of a 32-sphere tile and all lanes
//      stream the same static geometry (a shared-memory broadcast): static
//      spheres, axis-aligned boxes, rotated boxes, capsules, then the tile's
//      moving-sphere partners (self pairs, lane masks). Remaining pairs run in
//      type-uniform segments, one pair per lane. A warp vote every few
//      geometries stops the sweep at the first colliding pair.
// The static tables are staged into shared memory once per block by a bulk
// (TMA) copy; every wait on it is bounded and reports through p.status.
#pragma once
#include <algorithm>

#include <cfloat>

#include "csd_internal.h"

namespace csd {

constexpr unsigned kFull = 0xffffffffu;
constexpr long long kSpinLimit = 1ll << 26;   // mbarrier polls before a wait gives up
constexpr int kStaticSmemLimit = 96 * 1024;   // larger static tables are read from global memory
constexpr int kWarpsPerBlock = 8;

struct VoxArgs {
  const float* vox;
  int nv;
  float vr;
  const uint32_t* tile_mask;
  const uint32_t* other;
  int num_other;
  // voxel hash grid (voxgrid.cu); gstart == nullptr: every voxel is tested
  const float4* gvox;   // voxels ordered by bucket
  const int* gstart;    // [buckets + 1] first voxel of each bucket
  int gmask;            // buckets - 1 (a power of two minus one)
  float ginv_h;         // 1 / cell edge
};

static inline VoxArgs vox_args(const VoxelTables& vt) {
  return VoxArgs{vt.vox, vt.nv, vt.vr, vt.tile_mask, vt.other, vt.num_other, vt.gvox, vt.gstart, vt.gmask, vt.ginv_h};
}

// ---- voxel hash grid: cell (floor(x/h), floor(y/h), floor(z/h)) computed as
// floor(x * inv_h), which is monotone in x, so a voxel within R of a point
// lies in a cell between the cells of the point -/+ R on every axis. Buckets
// by the spatial hash of Teschner et al. (2003), "Optimized Spatial Hashing
// for Collision Detection of Deformable Objects" (primes 73856093, 19349663,
// 83492791); cells sharing a bucket only add candidates.
static __host__ __device__ __forceinline__ int vox_cell(float x, float inv_h) {
#ifdef __CUDA_ARCH__
  return __float2int_rd(__fmul_rn(x, inv_h));
#else
  const float v = floorf(x * inv_h);
  return v >= 2147483520.f ? 2147483520 : v <= -2147483520.f ? -2147483520 : (int)v;
#endif
}
static __host__ __device__ __forceinline__ uint32_t vox_bucket(int ix, int iy, int iz, int mask) {
  return ((uint32_t)ix * 73856093u ^ (uint32_t)iy * 19349663u ^ (uint32_t)iz * 83492791u) & (uint32_t)mask;
}
constexpr int kVoxGridMaxCells = 512;   // larger query boxes test every voxel
constexpr int kVoxGridMinVoxels = 64;   // fewer voxels are tested without a grid

// Per-warp shared memory (floats): slot transforms [slots][12], the warp's
// configuration [kMaxDim], two spare configurations (edge endpoints)
// [2][kMaxDim], moving world poses [pose_words].
static __host__ __device__ __forceinline__ int warp_floats(const DevPlant& p) {
  return p.num_slots * 12 + 3 * kMaxDim + ((p.pose_words + 3) & ~3);
}

// ------------------------------------------------------------ bulk staging
static __device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// Copies the static tables (p.static_bytes, a multiple of 16) into dst with
// one cp.async.bulk per 64 KiB chunk completing on an mbarrier, then
// invalidates the barrier so a later call can stage another plant. Returns
// false (and sets p.status) if the wait does not complete within kSpinLimit
// polls. Every thread of the block must call it.
// Polls an mbarrier phase at most `limit` times; 1 when it completed.
static __device__ __forceinline__ unsigned poll_mbarrier(uint64_t* bar, unsigned parity, long long limit) {
  unsigned done = 0;
  for (long long i = 0; i < limit && !done; ++i)
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
  return done;
}

static __device__ bool stage_statics(const DevPlant& p, float4* dst, uint64_t* bar) {
  const unsigned bytes = (unsigned)p.static_bytes;
  if (bytes == 0) return true;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    const char* src = reinterpret_cast<const char*>(p.statics);
    char* d = reinterpret_cast<char*>(dst);
    for (unsigned off = 0; off < bytes; off += 65536u) {
      unsigned n = min(65536u, bytes - off);
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(d + off)),
          "l"(src + off), "r"(n), "r"(smem_addr(bar))
          : "memory");
    }
  }
  __syncthreads();
  const unsigned done = poll_mbarrier(bar, 0, kSpinLimit);
  // block-uniform outcome: every thread has seen the phase complete, or the block gives up together
  if (!__syncthreads_and(done)) {
    if (threadIdx.x == 0) atomicExch(p.status, 1);
    // wait (bounded) once more for the copy still in flight before the block leaves
    poll_mbarrier(bar, 0, kSpinLimit);
    return false;
  }
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
  return true;
}

// Self-test of the bounded wait and its reporting: an mbarrier expecting 16
// bytes that no copy ever delivers, polled `limit` times; the block then gives
// up exactly as stage_statics does and sets the plant's status word. No
// asynchronous operation is in flight when the block leaves.
static __global__ void staging_wait_selftest_kernel(int* status, long long limit) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)), "r"(16u)
                 : "memory");
  }
  __syncthreads();
  const unsigned done = poll_mbarrier(&bar, 0, limit);
  if (!__syncthreads_and(done) && threadIdx.x == 0) atomicExch(status, 1);
}

// ---------------------------------------------------------------------- FK
// FK of the configuration in qs (shared, dim floats) into X[slot][12].
static __device__ __forceinline__ void fk_warp(const DevPlant& p, const float* qs, float* X, int lane) {
  float sj = 0.f, cj = 1.f, qj = 0.f;
  if (lane < p.num_fk) {
    qj = qs[__ldg(&p.fk[lane].qidx)];
    sincosf(qj, &sj, &cj);
  }
  const int r = lane < 9 ? lane % 3 : lane - 9;
  const int base = lane < 9 ? (lane / 3) * 3 : 9;
  for (int j = 0; j < p.num_fk; ++j) {
    const FkJoint* J = p.fk + j;
    const int type = __ldg(&J->type), parent = __ldg(&J->parent), child = __ldg(&J->child);
    const float s = __shfl_sync(kFull, sj, j), c = __shfl_sync(kFull, cj, j), qv = __shfl_sync(kFull, qj, j);
    float loc = 0.f;
    if (lane < 9) {
      float P = __ldg(&J->P[lane]);
      loc = type == J_REVOLUTE ? fmaf(c, P, fmaf(s, __ldg(&J->S[lane]), __ldg(&J->T[lane]))) : P;
    } else if (lane < 12) {
      float t = __ldg(&J->t[lane - 9]);
      loc = type == J_PRISMATIC ? fmaf(__ldg(&J->v[lane - 9]), qv, t) : t;
    }
    float out = loc;
    if (parent >= 0) {
      const float a0 = __shfl_sync(kFull, loc, base);
      const float a1 = __shfl_sync(kFull, loc, base + 1);
      const float a2 = __shfl_sync(kFull, loc, base + 2);
      if (lane < 12) {
        const float* Xp = X + parent * 12;
        float acc = lane < 9 ? Xp[r] * a0 : fmaf(Xp[r], a0, Xp[9 + r]);
        acc = fmaf(Xp[3 + r], a1, acc);
        out = fmaf(Xp[6 + r], a2, acc);
      }
    }
    __syncwarp();
    if (lane < 12) X[child * 12 + lane] = out;
    __syncwarp();
  }
}

// ---------------------------------------------------------------- placement
static __device__ __forceinline__ int pose_offset(const DevPlant& p, int m) {
  if (m < p.num_msph) return 4 * m;
  if (m < p.num_msph + p.num_mcap) return 4 * p.num_msph + 8 * (m - p.num_msph);
  return 4 * p.num_msph + 8 * p.num_mcap + 16 * (m - p.num_msph - p.num_mcap);
}

static __device__ __forceinline__ void place_all(const DevPlant& p, const float* X, float* pose, int lane) {
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
    const float* src = X + g.slot * 12;
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = src[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) t[i] = src[9 + i];
    float out[16];
    place_moving(g, R, t, out);
    float* dst = pose + g.pose_off;
    int nw = g.type == G_SPHERE ? 4 : g.type == G_CAPSULE ? 8 : 16;
    for (int i = 0; i < nw; i += 4)
      *reinterpret_cast<float4*>(dst + i) = make_float4(out[i], out[i + 1], out[i + 2], out[i + 3]);
  }
}

static __device__ __forceinline__ void load4f(const float4* src, int nq, float* out) {
  for (int i = 0; i < nq; ++i) {
    float4 v = src[i];
    out[4 * i] = v.x;
    out[4 * i + 1] = v.y;
    out[4 * i + 2] = v.z;
    out[4 * i + 3] = v.w;
  }
}

static __device__ __forceinline__ void own_sphere(const DevPlant& p, const float* pose, int m, float* c) {
  if (m < p.num_msph) {
    float4 v = *reinterpret_cast<const float4*>(pose + 4 * m);
    c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
  } else {  // no sphere: far away, tests report free
    c[0] = c[1] = c[2] = 1e30f;
    c[3] = 0.f;
  }
}

// ------------------------------------------------------------ broad phase
// Link-level culling of one configuration. Lane k (< num_slots) places its
// slot's bounding sphere in the world; `link` (lane k) has bit j set when the
// spheres of slots k and j overlap, `stat` (lane g) has bit i set when static
// 32 g + i overlaps some slot sphere. Statics are tested in groups of 32: the
// slots whose spheres overlap the group's sphere are found by one ballot, and
// each static of the group is tested against those slots only (none: the
// group is culled without a static test); a slot that cannot reach any static
// of the group in any configuration (host reach masks) is not among them. The
// spheres are padded on the host
// (the group spheres once more), so a culled pair is separated by at least
// 1e-4 m. With culling off every bit is set.
struct Cull {
  uint32_t link;
  uint32_t stat;
  const uint8_t* msl;  // slot of each moving geometry (staged copy)
};

static __device__ __forceinline__ Cull broad_phase(const DevPlant& p, const float4* aabb, const float* X, int lane) {
  // the staged region continues after the aligned boxes: static spheres, slot spheres, geometry slots
  const float4* sbs = aabb + 2 * p.num_sabox;
  const float4* slb = sbs + p.num_static;
  const float4* gbs = slb + p.num_slots;
  const int ng = (p.num_static + kWarp - 1) / kWarp;
  const uint32_t* gmk = reinterpret_cast<const uint32_t*>(gbs + ng);  // per group: slots that can reach it
  Cull c{~0u, ~0u, reinterpret_cast<const uint8_t*>(gmk + ((ng + 3) & ~3))};
  if (!p.cull) return c;
  float cx = 0.f, cy = 0.f, cz = 0.f, cr = -1.f;
  if (lane < p.num_slots) {
    const float4 b = slb[lane];
    const float* x = X + lane * 12;
    cx = fmaf(x[6], b.z, fmaf(x[3], b.y, fmaf(x[0], b.x, x[9])));
    cy = fmaf(x[7], b.z, fmaf(x[4], b.y, fmaf(x[1], b.x, x[10])));
    cz = fmaf(x[8], b.z, fmaf(x[5], b.y, fmaf(x[2], b.x, x[11])));
    cr = b.w;
  }
  uint32_t lw = 0;
  for (int j = 0; j < p.num_slots; ++j) {
    const float ox = __shfl_sync(kFull, cx, j), oy = __shfl_sync(kFull, cy, j), oz = __shfl_sync(kFull, cz, j);
    const float orr = __shfl_sync(kFull, cr, j);
    const float dx = cx - ox, dy = cy - oy, dz = cz - oz, t = cr + orr;
    // !(d2 > t2): a NaN pose counts as near, so its pairs are tested (and collide) as in the full sweep
    if (cr >= 0.f && orr >= 0.f && !(fmaf(dz, dz, fmaf(dy, dy, dx * dx)) > t * t)) lw |= 1u << j;
  }
  c.link = lw;
  uint32_t sw = 0;
  for (int g = 0; g * kWarp < p.num_static; ++g) {
    const float4 B = gbs[g];
    const float bx = cx - B.x, by = cy - B.y, bz = cz - B.z, bt = cr + B.w;
    // a slot that cannot reach the group is skipped (unless its pose is NaN, which is near everything)
    const bool reach = ((gmk[g] >> lane) & 1u) || !(cx == cx && cy == cy && cz == cz);
    uint32_t km = __ballot_sync(kFull, cr >= 0.f && B.w >= 0.f && reach &&
                                           !(fmaf(bz, bz, fmaf(by, by, bx * bx)) > bt * bt));
    uint32_t bits = 0u;
    if (km) {  // uniform across the warp
      const int st = g * kWarp + lane;
      float4 S = make_float4(0.f, 0.f, 0.f, -1.f);
      if (st < p.num_static) S = sbs[st];
      bool near = false;
      while (km) {
        const int k = __ffs(km) - 1;
        km &= km - 1u;
        const float kx = __shfl_sync(kFull, cx, k), ky = __shfl_sync(kFull, cy, k), kz = __shfl_sync(kFull, cz, k);
        const float kr = __shfl_sync(kFull, cr, k);
        const float dx = kx - S.x, dy = ky - S.y, dz = kz - S.z, t = kr + S.w;
        near |= S.w >= 0.f && !(fmaf(dz, dz, fmaf(dy, dy, dx * dx)) > t * t);
      }
      bits = __ballot_sync(kFull, near);
    }
    if (lane == g) sw = bits;
  }
  c.stat = sw;
  return c;
}

// Flag bit of static s (every lane may ask for a different s; all lanes call).
static __device__ __forceinline__ bool static_near(const Cull& c, int s) {
  return (__shfl_sync(kFull, c.stat, (s >> 5) & 31) >> (s & 31)) & 1u;
}

// Flag bits of statics [w0, w0 + 32) restricted to [lo, hi) (w0 a multiple of 32).
static __device__ __forceinline__ uint32_t near_bits(const Cull& c, int w0, int lo, int hi) {
  uint32_t b = __shfl_sync(kFull, c.stat, (w0 >> 5) & 31);
  if (lo > w0) b &= ~((1u << (lo - w0)) - 1u);
  if (hi - w0 < 32) b &= (1u << (hi - w0)) - 1u;
  return b;
}

// ------------------------------------------------------------------- sweeps
// Tile t (moving spheres 32t .. 32t+31) against its static geometries and
// moving-sphere partners. Returns the warp-uniform "some pair collides".
static __device__ bool sweep_tile(const DevPlant& p, const float4* stat, const float4* aabb, const float* pose, int t,
                                  int lane, bool skip_dense, const Cull& cu) {
  const TileInfo ti = p.tiles[t];
  float c[4];
  own_sphere(p, pose, t * kWarp + lane, c);
  const float r2 = c[3] * c[3];
  bool hit = false;
  const int s0 = 0, s1 = p.num_ssph, s2 = s1 + p.num_sabox, s3 = s2 + p.num_srbox, s4 = s3 + p.num_scap;
  // static spheres (with skip_dense: swept with the aligned boxes by sweep_dense_spheres)
  if (skip_dense) {
  } else if (ti.dense[SC_SPH]) {
    int s = s0;
    for (; s + 8 <= s1; s += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const float4 S = stat[4 * (s + u)];
        const float d0 = c[0] - S.x, d1 = c[1] - S.y, d2 = c[2] - S.z;
        const float dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
        const float rr = c[3] + S.w;
        hit |= !(dd >= rr * rr);
      }
      if (__any_sync(kFull, hit)) return true;
    }
    for (; s < s1; ++s) {
      const float4 S = stat[4 * s];
      const float d0 = c[0] - S.x, d1 = c[1] - S.y, d2 = c[2] - S.z;
      const float dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
      const float rr = c[3] + S.w;
      hit |= !(dd >= rr * rr);
    }
  } else {
    for (int e = ti.ent[SC_SPH]; e < ti.ent[SC_SPH + 1]; ++e) {
      TileEntry en = p.entries[e];
      if (!static_near(cu, (int)en.s)) continue;
      float4 S = stat[4 * en.s];
      float d0 = c[0] - S.x, d1 = c[1] - S.y, d2 = c[2] - S.z;
      float dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
      float rr = c[3] + S.w;
      hit |= ((en.mask >> lane) & 1u) && !(dd >= rr * rr);
      if ((e & 7) == 7 && __any_sync(kFull, hit)) return true;
    }
  }
  if (__any_sync(kFull, hit)) return true;
  // axis-aligned static boxes
  if (skip_dense) {
  } else if (ti.dense[SC_ABOX]) {
    int i = 0;
    for (; i + 8 <= p.num_sabox; i += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) hit |= sph_abox_hit(c, c[3], aabb[2 * (i + u)], aabb[2 * (i + u) + 1]);
      if (__any_sync(kFull, hit)) return true;
    }
    for (; i < p.num_sabox; ++i) hit |= sph_abox_hit(c, c[3], aabb[2 * i], aabb[2 * i + 1]);
  } else {
    for (int e = ti.ent[SC_ABOX]; e < ti.ent[SC_ABOX + 1]; ++e) {
      TileEntry en = p.entries[e];
      if (!static_near(cu, (int)en.s)) continue;
      const int i = en.s - s1;
      hit |= ((en.mask >> lane) & 1u) && sph_abox_hit(c, c[3], aabb[2 * i], aabb[2 * i + 1]);
      if ((e & 7) == 7 && __any_sync(kFull, hit)) return true;
    }
  }
  if (__any_sync(kFull, hit)) return true;
  // rotated static boxes
  for (int k = 0, e = ti.ent[SC_RBOX]; ti.dense[SC_RBOX] ? k < s3 - s2 : e < ti.ent[SC_RBOX + 1]; ++k, ++e) {
    int s = s2 + k;
    uint32_t mask = kFull;
    if (!ti.dense[SC_RBOX]) {
      TileEntry en = p.entries[e];
      s = en.s;
      mask = en.mask;
    }
    if (!static_near(cu, s)) continue;
    float B[16];
    load4f(stat + 4 * s, 4, B);
    hit |= ((mask >> lane) & 1u) && sph_box_hit(c, c[3], B);
    if ((k & 3) == 3 && __any_sync(kFull, hit)) return true;
  }
  // static capsules
  for (int k = 0, e = ti.ent[SC_CAP]; ti.dense[SC_CAP] ? k < s4 - s3 : e < ti.ent[SC_CAP + 1]; ++k, ++e) {
    int s = s3 + k;
    uint32_t mask = kFull;
    if (!ti.dense[SC_CAP]) {
      TileEntry en = p.entries[e];
      s = en.s;
      mask = en.mask;
    }
    if (!static_near(cu, s)) continue;
    float C[8];
    load4f(stat + 4 * s, 2, C);
    hit |= ((mask >> lane) & 1u) && sph_cap_hit(c, C);
    if ((k & 3) == 3 && __any_sync(kFull, hit)) return true;
  }
  if (__any_sync(kFull, hit)) return true;
  // moving-sphere partners
  for (int e = ti.self_begin; e < ti.self_end; ++e) {
    TileEntry en = p.entries[e];
    float4 Q = *reinterpret_cast<const float4*>(pose + 4 * en.s);
    float d0 = c[0] - Q.x, d1 = c[1] - Q.y, d2 = c[2] - Q.z;
    float dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
    float rr = c[3] + Q.w;
    hit |= ((en.mask >> lane) & 1u) && !(dd >= rr * rr);
    if ((e & 7) == 7 && __any_sync(kFull, hit)) return true;
  }
  (void)r2;
  return __any_sync(kFull, hit);
}

// NaN-propagating minimum (a NaN distance counts as a collision, as in the
// compare-based tests).
static __device__ __forceinline__ float fmin_nan(float a, float b) {
  float r;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Moving spheres against the static spheres and axis-aligned boxes when every
// tile is dense for both classes: lane holds spheres lane, lane + 32, ...
// (R of them), so each broadcast static feeds R tests. A pair collides iff
// d^2 - (r_a + r_b)^2 < 0 (one rounding, by FMA) and hits accumulate as a
// NaN-propagating minimum voted every 8 statics.
template <int R>
static __device__ bool sweep_dense_spheres(const DevPlant& p, const float4* stat, const float4* aabb, const float* pose,
                                           int lane, const Cull& cu) {
  float cx[R], cy[R], cz[R], cr[R];
#pragma unroll
  for (int j = 0; j < R; ++j) {
    float c[4];
    own_sphere(p, pose, j * kWarp + lane, c);
    cx[j] = c[0];
    cy[j] = c[1];
    cz[j] = c[2];
    cr[j] = c[3];
  }
  float m = FLT_MAX;
  int cnt = 0;
  const int ns = p.num_ssph, nb = p.num_sabox;
  for (int w0 = 0; w0 < ns; w0 += kWarp) {
    uint32_t bits = near_bits(cu, w0, 0, ns);
    while (bits) {
      const int st = w0 + __ffs(bits) - 1;
      bits &= bits - 1u;
      const float4 S = stat[4 * st];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const float d0 = cx[j] - S.x, d1 = cy[j] - S.y, d2 = cz[j] - S.z;
        const float dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
        const float rr = cr[j] + S.w;
        m = fmin_nan(m, fmaf(-rr, rr, dd));
      }
      if ((++cnt & 7) == 0 && __any_sync(kFull, !(m >= 0.f))) return true;
    }
  }
  if (__any_sync(kFull, !(m >= 0.f))) return true;
  for (int w0 = ns & ~(kWarp - 1); w0 < ns + nb; w0 += kWarp) {
    uint32_t bits = near_bits(cu, w0, ns, ns + nb);
    while (bits) {
      const int i = w0 + __ffs(bits) - 1 - ns;
      bits &= bits - 1u;
      const float4 P = aabb[2 * i], H = aabb[2 * i + 1];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const float e0 = fmaxf(fabsf(cx[j] - P.x) - H.x, 0.f);
        const float e1 = fmaxf(fabsf(cy[j] - P.y) - H.y, 0.f);
        const float e2 = fmaxf(fabsf(cz[j] - P.z) - H.z, 0.f);
        const float ee = fmaf(e2, e2, fmaf(e1, e1, e0 * e0));
        m = fmin_nan(m, fmaf(-cr[j], cr[j], ee));
      }
      if ((++cnt & 7) == 0 && __any_sync(kFull, !(m >= 0.f))) return true;
    }
  }
  return __any_sync(kFull, !(m >= 0.f));
}

template <int T>
struct Words {
  static constexpr int n = T == G_SPHERE ? 4 : T == G_CAPSULE ? 8 : 16;
};

// One type-uniform segment of generic pairs, one pair per lane.
// Whether a generic pair survives the broad phase: its static is near some
// link, or its two moving geometries' link spheres overlap (all lanes call).
template <bool BSTATIC>
static __device__ __forceinline__ bool pair_near(const DevPlant& p, const Cull& cu, const GenericPair& gp, bool valid) {
  if (BSTATIC) return static_near(cu, valid ? (int)(gp.b & 0x7fffffffu) : 0) && valid;
  const int sa = valid ? (int)cu.msl[gp.a] : 0, sb = valid ? (int)cu.msl[gp.b] : 0;
  return ((__shfl_sync(kFull, cu.link, sa & 31) >> (sb & 31)) & 1u) && valid;
}

template <int TA, int TB, bool BSTATIC>
static __device__ bool generic_segment(const DevPlant& p, const float4* stat, const float* pose, const GenSeg& sg,
                                       int lane, const Cull& cu) {
  // the next pass's pair indices are loaded one pass ahead (their latency
  // would otherwise stall every pass)
  GenericPair nxt{0u, 0u};
  if (sg.begin + lane < sg.end) nxt = p.generic[sg.begin + lane];
  for (int base = sg.begin; base < sg.end; base += kWarp) {
    const int k = base + lane;
    const GenericPair gp = nxt;
    if (k + kWarp < sg.end) nxt = p.generic[k + kWarp];
    const bool keep = pair_near<BSTATIC>(p, cu, gp, k < sg.end);
    if (!__any_sync(kFull, keep)) continue;
    bool hit = false;
    if (keep) {
      float A[Words<TA>::n], B[Words<TB>::n];
      const float4* pa = reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.a));
#pragma unroll
      for (int i = 0; i < Words<TA>::n / 4; ++i) {
        float4 v = pa[i];
        A[4 * i] = v.x; A[4 * i + 1] = v.y; A[4 * i + 2] = v.z; A[4 * i + 3] = v.w;
      }
      const float4* pb = BSTATIC ? stat + 4 * (gp.b & 0x7fffffffu)
                                 : reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.b));
#pragma unroll
      for (int i = 0; i < Words<TB>::n / 4; ++i) {
        float4 v = pb[i];
        B[4 * i] = v.x; B[4 * i + 1] = v.y; B[4 * i + 2] = v.z; B[4 * i + 3] = v.w;
      }
      hit = pair_hit(TA, A, TB, B);
    }
    if (__any_sync(kFull, hit)) return true;
  }
  return false;
}

// One moving-moving segment by link-pair runs: lane r takes run r of a chunk
// of 32 and reads the overlap bit of its two slots; the warp then sweeps the
// pairs of each stretch of consecutive overlapping runs (adjacent in the pair
// list) as one range, one pair per lane. A run of culled slots costs no
// pair-index load and no per-pair test; with culling off a chunk is one range.
template <int TA, int TB>
static __device__ bool generic_runs(const DevPlant& p, const float* pose, const GenSeg& sg, int lane,
                                    const Cull& cu) {
  for (int r0 = sg.run_begin; r0 < sg.run_end; r0 += kWarp) {
    const int r = r0 + lane;
    PairRun pr{0, 0, 0, 0};
    if (r < sg.run_end) pr = p.runs[r];
    const bool keep = ((__shfl_sync(kFull, cu.link, pr.sa & 31) >> (pr.sb & 31)) & 1u) && r < sg.run_end;
    uint32_t km = __ballot_sync(kFull, keep);
    while (km) {
      const int j = __ffs(km) - 1;
      const uint32_t t = km >> j;  // the stretch of set bits from j
      const int len = t == 0xffffffffu ? kWarp : __ffs(~t) - 1;
      km = len == kWarp ? 0u : km & ~(((1u << len) - 1u) << j);
      const int b0 = __shfl_sync(kFull, pr.begin, j), b1 = __shfl_sync(kFull, pr.end, j + len - 1);
      for (int base = b0; base < b1; base += kWarp) {
        const int k = base + lane;
        bool hit = false;
        if (k < b1) {
          const GenericPair gp = p.generic[k];
          float A[Words<TA>::n], B[Words<TB>::n];
          const float4* pa = reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.a));
#pragma unroll
          for (int i = 0; i < Words<TA>::n / 4; ++i) {
            float4 v = pa[i];
            A[4 * i] = v.x; A[4 * i + 1] = v.y; A[4 * i + 2] = v.z; A[4 * i + 3] = v.w;
          }
          const float4* pb = reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.b));
#pragma unroll
          for (int i = 0; i < Words<TB>::n / 4; ++i) {
            float4 v = pb[i];
            B[4 * i] = v.x; B[4 * i + 1] = v.y; B[4 * i + 2] = v.z; B[4 * i + 3] = v.w;
          }
          hit = pair_hit(TA, A, TB, B);
        }
        if (__any_sync(kFull, hit)) return true;
      }
    }
  }
  return false;
}

// Capsule x box segment with a broad phase: a lane tests its pair's capsule
// bounding sphere (centre, radius + half length) against the box; pairs that
// pass are compacted into a warp-wide batch (lane r of the batch holds the
// r-th candidate) and the exact segment-box test runs on full batches.
template <bool BSTATIC>
static __device__ bool cap_box_exact(const DevPlant& p, const float4* stat, const float* pose, int k) {
  bool hit = false;
  if (k >= 0) {
    const GenericPair gp = p.generic[k];
    float A[8], B[16];
    const float4* pa = reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.a));
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      float4 v = pa[i];
      A[4 * i] = v.x; A[4 * i + 1] = v.y; A[4 * i + 2] = v.z; A[4 * i + 3] = v.w;
    }
    const float4* pb = BSTATIC ? stat + 4 * (gp.b & 0x7fffffffu)
                               : reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.b));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float4 v = pb[i];
      B[4 * i] = v.x; B[4 * i + 1] = v.y; B[4 * i + 2] = v.z; B[4 * i + 3] = v.w;
    }
    hit = cap_box_hit(A, B);
  }
  return __any_sync(kFull, hit);
}

template <bool BSTATIC>
static __device__ bool cap_box_segment(const DevPlant& p, const float4* stat, const float* pose, const GenSeg& sg,
                                       int lane, const Cull& cu) {
  int pend = -1;  // pair index this lane holds in the pending batch
  int npend = 0;  // warp-uniform batch fill
  GenericPair nxt{0u, 0u};
  if (sg.begin + lane < sg.end) nxt = p.generic[sg.begin + lane];
  for (int base = sg.begin; base < sg.end; base += kWarp) {
    const int k = base + lane;
    const GenericPair gp = nxt;
    if (k + kWarp < sg.end) nxt = p.generic[k + kWarp];
    const bool keep = pair_near<BSTATIC>(p, cu, gp, k < sg.end);
    bool cand = false;
    if (keep) {
      const int oa = pose_offset(p, (int)gp.a);
      const float4 ca = *reinterpret_cast<const float4*>(pose + oa);
      const float hl = pose[oa + 7];
      const float4* pb = BSTATIC ? stat + 4 * (gp.b & 0x7fffffffu)
                                 : reinterpret_cast<const float4*>(pose + pose_offset(p, (int)gp.b));
      float B[16];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        float4 v = pb[i];
        B[4 * i] = v.x; B[4 * i + 1] = v.y; B[4 * i + 2] = v.z; B[4 * i + 3] = v.w;
      }
      const float c[3] = {ca.x, ca.y, ca.z};
      cand = sph_box_hit(c, ca.w + hl, B);
    }
    const unsigned m = __ballot_sync(kFull, cand);
    const int cnt = __popc(m);
    const int take = min(cnt, kWarp - npend);
    const int r = lane - npend;
    const int src = (r >= 0 && r < take) ? (int)__fns(m, 0, r + 1) : 0;
    const int kk = __shfl_sync(kFull, k, src);
    if (r >= 0 && r < take) pend = kk;
    npend += take;
    if (npend == kWarp) {
      if (cap_box_exact<BSTATIC>(p, stat, pose, pend)) return true;
      const int over = cnt - take;
      const int src2 = lane < over ? (int)__fns(m, 0, take + lane + 1) : 0;
      const int k2 = __shfl_sync(kFull, k, src2);
      pend = lane < over ? k2 : -1;
      npend = over;
    }
  }
  if (npend > 0) return cap_box_exact<BSTATIC>(p, stat, pose, lane < npend ? pend : -1);
  return false;
}

// Remaining pairs (the moving geometry first; moving-moving pairs ordered
// sphere < capsule < box), dispatched once per segment.
static __device__ bool sweep_generic(const DevPlant& p, const float4* stat, const float* pose, int lane,
                                     const Cull& cu) {
  for (int sgi = 0; sgi < p.num_segs; ++sgi) {
    const GenSeg sg = p.segs[sgi];
    const int key = sg.b_static * 16 + sg.ta * 4 + sg.tb;
    bool h = false;
    switch (key) {
      // moving-moving
      case G_SPHERE * 4 + G_CAPSULE: h = generic_runs<G_SPHERE, G_CAPSULE>(p, pose, sg, lane, cu); break;
      case G_SPHERE * 4 + G_BOX: h = generic_runs<G_SPHERE, G_BOX>(p, pose, sg, lane, cu); break;
      case G_CAPSULE * 4 + G_CAPSULE: h = generic_runs<G_CAPSULE, G_CAPSULE>(p, pose, sg, lane, cu); break;
      case G_CAPSULE * 4 + G_BOX: h = cap_box_segment<false>(p, stat, pose, sg, lane, cu); break;
      case G_BOX * 4 + G_BOX: h = generic_runs<G_BOX, G_BOX>(p, pose, sg, lane, cu); break;
      case G_BOX * 4 + G_SPHERE: h = generic_runs<G_BOX, G_SPHERE>(p, pose, sg, lane, cu); break;
      case G_BOX * 4 + G_CAPSULE: h = generic_runs<G_BOX, G_CAPSULE>(p, pose, sg, lane, cu); break;
      case G_CAPSULE * 4 + G_SPHERE: h = generic_runs<G_CAPSULE, G_SPHERE>(p, pose, sg, lane, cu); break;
      case G_SPHERE * 4 + G_SPHERE: h = generic_runs<G_SPHERE, G_SPHERE>(p, pose, sg, lane, cu); break;
      // moving-static
      case 16 + G_CAPSULE * 4 + G_SPHERE: h = generic_segment<G_CAPSULE, G_SPHERE, true>(p, stat, pose, sg, lane, cu); break;
      case 16 + G_CAPSULE * 4 + G_BOX: h = cap_box_segment<true>(p, stat, pose, sg, lane, cu); break;
      case 16 + G_CAPSULE * 4 + G_CAPSULE: h = generic_segment<G_CAPSULE, G_CAPSULE, true>(p, stat, pose, sg, lane, cu); break;
      case 16 + G_BOX * 4 + G_SPHERE: h = generic_segment<G_BOX, G_SPHERE, true>(p, stat, pose, sg, lane, cu); break;
      case 16 + G_BOX * 4 + G_BOX: h = generic_segment<G_BOX, G_BOX, true>(p, stat, pose, sg, lane, cu); break;
      case 16 + G_BOX * 4 + G_CAPSULE: h = generic_segment<G_BOX, G_CAPSULE, true>(p, stat, pose, sg, lane, cu); break;
      default: h = generic_segment<G_SPHERE, G_SPHERE, true>(p, stat, pose, sg, lane, cu); break;
    }
    if (h) return true;
  }
  return false;
}

// Voxels near one geometry through the hash grid: every voxel in the cells
// covering the geometry's bounding sphere (bc, br) grown by the voxel radius
// (x 1.001 + 1e-4 m, above any FP32 rounding of the pair tests) is tested
// with the same pair test as the full sweep, so the verdict is the full
// sweep's. SPH: the geometry is the sphere G (tested as in the tile sweep).
template <bool SPH>
static __device__ bool grid_geom_hit(const VoxArgs& va, int tg, const float* G, const float* bc, float br) {
  const float R = __fmaf_rn(__fadd_rn(br, va.vr), 1.001f, 1e-4f);
  int lo[3], hi[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lo[i] = vox_cell(__fsub_rn(bc[i], R), va.ginv_h);
    hi[i] = vox_cell(__fadd_rn(bc[i], R), va.ginv_h);
  }
  const long long cells = (long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
  const bool finite = isfinite(bc[0]) && isfinite(bc[1]) && isfinite(bc[2]) && isfinite(R);
  if (!finite || cells > kVoxGridMaxCells) {  // (a NaN pose collides with every voxel in the full sweep)
    for (int v = 0; v < va.nv; ++v) {
      float S[4] = {__ldg(va.vox + 3 * v), __ldg(va.vox + 3 * v + 1), __ldg(va.vox + 3 * v + 2), va.vr};
      if (SPH ? sph_sph_hit(G, S) : pair_hit(G_SPHERE, S, tg, G)) return true;
    }
    return false;
  }
  for (int ix = lo[0]; ix <= hi[0]; ++ix)
    for (int iy = lo[1]; iy <= hi[1]; ++iy)
      for (int iz = lo[2]; iz <= hi[2]; ++iz) {
        const uint32_t b = vox_bucket(ix, iy, iz, va.gmask);
        const int k1 = __ldg(va.gstart + b + 1);
        for (int k = __ldg(va.gstart + b); k < k1; ++k) {
          const float4 v = __ldg(va.gvox + k);
          float S[4] = {v.x, v.y, v.z, va.vr};
          if (SPH ? sph_sph_hit(G, S) : pair_hit(G_SPHERE, S, tg, G)) return true;
        }
      }
  return false;
}

// Bounding sphere of a world-posed geometry (WG layout: sphere [c r],
// capsule [a r | u hl], box [x -q0 | y -q1 | z -q2 | h]).
static __device__ __forceinline__ float geom_bound(int tg, const float* G, float* c) {
  if (tg == G_SPHERE || tg == G_CAPSULE) {
    c[0] = G[0];
    c[1] = G[1];
    c[2] = G[2];
    return tg == G_SPHERE ? G[3] : G[3] + G[7];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) c[r] = -fmaf(G[8 + r], G[11], fmaf(G[4 + r], G[7], G[r] * G[3]));
  return sqrtf(fmaf(G[14], G[14], fmaf(G[13], G[13], G[12] * G[12])));
}

static __device__ bool sweep_voxels_grid(const DevPlant& p, const float4* stat, const float* pose, const VoxArgs& va,
                                         int lane) {
  for (int t = 0; t < p.num_tiles; ++t) {
    const uint32_t mask = va.tile_mask[t];
    if (!mask) continue;
    float c[4];
    own_sphere(p, pose, t * kWarp + lane, c);
    const bool hit = ((mask >> lane) & 1u) && grid_geom_hit<true>(va, G_SPHERE, c, c, c[3]);
    if (__any_sync(kFull, hit)) return true;
  }
  for (int o0 = 0; o0 < va.num_other; o0 += kWarp) {
    const int o = o0 + lane;
    bool hit = false;
    if (o < va.num_other) {
      const uint32_t ref = va.other[o];
      float G[16];
      int tg;
      if (ref & 0x80000000u) {
        const int s = (int)(ref & 0x7fffffffu);
        tg = __ldg(p.static_type + s);
        load4f(stat + 4 * s, tg == G_SPHERE ? 1 : tg == G_CAPSULE ? 2 : 4, G);
      } else {
        tg = __ldg(&p.moving[ref].type);
        const int nw = tg == G_SPHERE ? 4 : tg == G_CAPSULE ? 8 : 16;
        const float* src = pose + pose_offset(p, (int)ref);
        for (int i = 0; i < nw; ++i) G[i] = src[i];
      }
      float bc[3];
      const float br = geom_bound(tg, G, bc);
      hit = grid_geom_hit<false>(va, tg, G, bc, br);
    }
    if (__any_sync(kFull, hit)) return true;
  }
  return false;
}

static __device__ bool sweep_voxels(const DevPlant& p, const float4* stat, const float* pose, const VoxArgs& va,
                                    int lane) {
  if (va.gstart) return sweep_voxels_grid(p, stat, pose, va, lane);
  for (int t = 0; t < p.num_tiles; ++t) {
    const uint32_t mask = va.tile_mask[t];
    if (!mask) continue;
    float c[4];
    own_sphere(p, pose, t * kWarp + lane, c);
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
    const uint32_t ref = va.other[o];
    float G[16];
    int tg;
    if (ref & 0x80000000u) {
      const int s = (int)(ref & 0x7fffffffu);
      tg = __ldg(p.static_type + s);
      load4f(stat + 4 * s, tg == G_SPHERE ? 1 : tg == G_CAPSULE ? 2 : 4, G);
    } else {
      tg = __ldg(&p.moving[ref].type);
      const int nw = tg == G_SPHERE ? 4 : tg == G_CAPSULE ? 8 : 16;
      const float* src = pose + pose_offset(p, (int)ref);
      for (int i = 0; i < nw; ++i) G[i] = src[i];
    }
    for (int base = 0; base < va.nv; base += kWarp) {
      const int v = base + lane;
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

// Full check of the configuration whose slot transforms are in X
// (warp-uniform result: true = colliding).
static __device__ bool check_config(const DevPlant& p, const float4* stat, const float4* aabb, const float* X,
                                    float* pose, int lane, const VoxArgs& va) {
  __syncwarp();
  place_all(p, X, pose, lane);
  __syncwarp();
  if (p.always_colliding) return true;
  const Cull cu = broad_phase(p, aabb, X, lane);
  const bool dense = p.dense_spheres && p.num_tiles >= 1 && p.num_tiles <= 4;
  if (dense) {
    bool h;
    switch (p.num_tiles) {
      case 1: h = sweep_dense_spheres<1>(p, stat, aabb, pose, lane, cu); break;
      case 2: h = sweep_dense_spheres<2>(p, stat, aabb, pose, lane, cu); break;
      case 3: h = sweep_dense_spheres<3>(p, stat, aabb, pose, lane, cu); break;
      default: h = sweep_dense_spheres<4>(p, stat, aabb, pose, lane, cu); break;
    }
    if (h) return true;
  }
  for (int t = 0; t < p.num_tiles; ++t)
    if (sweep_tile(p, stat, aabb, pose, t, lane, dense, cu)) return true;
  if (sweep_generic(p, stat, pose, lane, cu)) return true;
  if (va.nv > 0 && sweep_voxels(p, stat, pose, va, lane)) return true;
  return false;
}

// Shared-memory setup common to the warp-per-configuration kernels. SM: the
// static tables are staged into shared memory.
template <bool SM>
struct WarpCtx {
  const float4* stat;
  const float4* aabb;
  float* X;
  float* qs;
  float* q1;
  float* q2;
  float* pose;
  bool ok;
};

template <bool SM>
static __device__ __forceinline__ WarpCtx<SM> warp_setup(const DevPlant& p, float4* smem4, uint64_t* bar) {
  WarpCtx<SM> w;
  const int warp = threadIdx.x >> 5;
  float* wbase;
  if (SM) {
    w.ok = stage_statics(p, smem4, bar);
    w.stat = smem4;
    w.aabb = smem4 + 4 * p.num_static;
    wbase = reinterpret_cast<float*>(smem4) + p.static_bytes / 4;
  } else {
    w.ok = true;
    w.stat = p.statics;
    w.aabb = p.aabb;
    wbase = reinterpret_cast<float*>(smem4);
  }
  w.X = wbase + warp * warp_floats(p);
  w.qs = w.X + p.num_slots * 12;
  w.q1 = w.qs + kMaxDim;
  w.q2 = w.q1 + kMaxDim;
  w.pose = w.q2 + kMaxDim;
  return w;
}

// ---- host helpers shared by the launchers
static inline bool statics_in_smem(const csd_plant_s* p) { return p->dp.static_bytes <= kStaticSmemLimit; }

static inline size_t smem_bytes(const csd_plant_s* p, int wpb) {
  size_t per = (size_t)warp_floats(p->dp) * sizeof(float) * wpb;
  return per + (statics_in_smem(p) ? (size_t)p->dp.static_bytes : 0);
}

template <typename K>
static csd_status_t grid_for(K kernel, size_t smem, int64_t work_warps, int* grid, int wpb) {
  int per_sm = 0;
  CSD_CUDA_TRY(raise_smem_limit(kernel, (int)smem));
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
