// csd_device.cuh -- device-side plant layout, forward kinematics, geometry
// placement and primitive-pair tests for the fused collision kernels.
//
// Layout produced by plant.cu (host preprocessing of a MinimalPlant):
//   * Only joints with a moving degree of freedom are evaluated per
//     configuration ("FK joints"). Every link is attached to a "slot": the
//     nearest ancestor link (inclusive) whose parent joint moves, or the world
//     (slot -1). Fixed-joint chains are pre-composed on the host in FP64, so
//     a fixed tool frame on a moving link costs nothing per configuration.
//   * Geometries on the world slot are "static": their world pose is computed
//     once on the host. All others are "moving", ordered spheres first, then
//     capsules, then boxes.
//   * A geometry's world pose is 16 floats ("WG" format):
//       sphere : [c0 c1 c2 r | - - - - | ...]
//       capsule: [a0 a1 a2 r | u0 u1 u2 hl | ...]      (segment a + t u, |t| <= hl)
//       box    : [x0 x1 x2 -q0 | y0 y1 y2 -q1 | z0 z1 z2 -q2 | h0 h1 h2 -]
//                with x,y,z the box axes in world and q_i = axis_i . centre,
//                so the centre-relative coordinates of a point c are axis_i.c - q_i.
//
// Contact rule: the reference GPU rule (cuda_geometry_utilities.h:16-125):
// a pair is free iff dist^2 >= (sum of radii)^2; boxes by the 15-axis SAT with
// a strict separation test. Capsules (no reference semantics) follow the same
// "free iff dist^2 >= r^2" rule on exact segment distances.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace csd {

enum : int { J_FIXED = 0, J_REVOLUTE = 1, J_PRISMATIC = 2 };
enum : int { G_BOX = 0, G_SPHERE = 1, G_CYLINDER = 2, G_CAPSULE = 3 };

constexpr int kMaxDim = 16;          // configuration variables per plant
constexpr int kMaxRegionFaces = 4096;  // faces of an EI-ZO region (the reference's MAX_NUM_FACES is 4000)
constexpr int kMaxSlots = 32;        // moving links evaluated per configuration
constexpr int kWarp = 32;

// One moving joint, 40 words. R(q) = cq * P + sq * S + T for revolute joints,
// R = P and t(q) = t + v q for prismatic joints; parent = slot or -1 (world).
struct FkJoint {
  int type, parent, child, qidx;
  float P[9], S[9], T[9];
  float t[3], v[3];
  float pad[3];
};
static_assert(sizeof(FkJoint) == 160, "FkJoint is 10 float4");

// A moving geometry in its slot frame, 24 words.
struct MovingGeom {
  int type, slot, pose_off, pad;
  float r, hl, pad2, pad3;
  float p[3];    // centre in slot frame
  float z[3];    // capsule axis in slot frame
  float R[9];    // box rotation (column-major) in slot frame
  float h[3];    // box half extents  -- (R,h) only used by boxes
  float pad4[2];
};
static_assert(sizeof(MovingGeom) == 112, "MovingGeom is 7 float4");

// Static geometry classes, in table order.
enum : int { SC_SPH = 0, SC_ABOX = 1, SC_RBOX = 2, SC_CAP = 3 };

struct GenericPair {  // a: moving index; b: bit 31 set = static geometry, low bits = index
  uint32_t a, b;
};

struct GenSeg {       // generic pairs [begin, end) share (type a, type b, b static)
  int begin, end, ta, tb;
  int b_static;
  int run_begin, run_end;  // moving-moving segments: link-pair runs [run_begin, run_end) of the segment
  int pad0;
};

struct PairRun {      // generic pairs [begin, end) whose moving geometries lie on slots sa and sb
  int begin, end, sa, sb;
};

struct TileInfo {     // moving spheres [32*t, 32*t+32) against static geometries
  int dense[4];       // per static class: every valid lane pairs with every static of the class
  int ent[5];         // otherwise entries [ent[c], ent[c+1]) of class c
  int self_begin, self_end;  // moving-sphere partners of the tile's lanes (self pairs)
  int pad;
};

struct TileEntry {    // one static geometry (or moving partner) and the lanes of the tile that pair with it
  uint32_t s;
  uint32_t mask;
};

// Plant description passed to kernels by value (pointers are device memory).
struct DevPlant {
  int dim;
  int num_fk;            // FK joints
  int num_slots;         // moving links
  int num_moving;        // moving geometries
  int num_msph;          // moving spheres (first in the moving list)
  int num_mcap;          // moving capsules (next)
  int num_tiles;         // ceil(num_msph / 32)
  int num_static;        // static geometries: spheres, aligned boxes, rotated boxes, capsules
  int num_ssph, num_sabox, num_srbox, num_scap;
  int num_generic;       // generic pairs
  int num_segs;          // generic segments
  int pose_words;        // words of moving world poses per configuration
  int always_colliding;  // a static-static pair collides
  int num_links;         // all links of the reference tree (FK output)
  int static_bytes;      // bytes of statics + aabb staged in shared memory (multiple of 16)
  int dense_spheres;     // every tile pairs every lane with every static sphere and aligned box
  int cull;              // link-level broad phase on (slot and static bounding spheres)
  const FkJoint* fk;
  const MovingGeom* moving;
  const float4* statics;       // [num_static][4] float4 (WG format); followed by aabb
  const float4* aabb;          // [num_sabox][2]: [p 0 | h 0] of axis-aligned static boxes; followed by
                               // [num_static] static bounding spheres (world centre, radius), the slot
                               // spheres, [ceil(num_static / 32)] group spheres (each enclosing the
                               // bounding spheres of statics 32 g .. 32 g + 31) and the geometry slots
                               // below (one staged region)
  const float4* slot_bs;       // [num_slots] bounding sphere of each slot's geometry (slot frame); radius < 0: none
  const uint8_t* moving_slot;  // [num_moving] slot of each moving geometry
  const int* static_type;      // [num_static]
  const TileInfo* tiles;
  const TileEntry* entries;
  const GenericPair* generic;
  const GenSeg* segs;
  const PairRun* runs;
  const int* link_slot;        // [num_links] slot of each reference link (-1 world, -2 unreachable)
  const float* link_fixed;     // [num_links][12] slot->link (R col-major 9, t 3); world links: world pose
  int* status;                 // device error word: nonzero after a bounded wait gave up
};

// ------------------------------------------------------------------ FK
// X (12 floats): R col-major [0..8], t [9..11]. World composition of a joint
// whose parent world transform is (Rp, tp):
//   R = Rp * Rl(q), t = Rp * tl + tp.
__device__ __forceinline__ void compose(const float* Rp, const float* tp, const float* Rl, const float* tl,
                                        float* R, float* t) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      R[c * 3 + r] = fmaf(Rp[6 + r], Rl[c * 3 + 2], fmaf(Rp[3 + r], Rl[c * 3 + 1], Rp[r] * Rl[c * 3]));
#pragma unroll
  for (int r = 0; r < 3; ++r) t[r] = fmaf(Rp[6 + r], tl[2], fmaf(Rp[3 + r], tl[1], fmaf(Rp[r], tl[0], tp[r])));
}

// Local joint transform for configuration value qv.
__device__ __forceinline__ void joint_local(const FkJoint& J, float qv, float* Rl, float* tl) {
  if (J.type == J_REVOLUTE) {
    float s, c;
    sincosf(qv, &s, &c);
#pragma unroll
    for (int i = 0; i < 9; ++i) Rl[i] = fmaf(c, J.P[i], fmaf(s, J.S[i], J.T[i]));
#pragma unroll
    for (int i = 0; i < 3; ++i) tl[i] = J.t[i];
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) Rl[i] = J.P[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) tl[i] = fmaf(J.v[i], qv, J.t[i]);
  }
}

// ------------------------------------------------------------- placement
// World pose of moving geometry g given its slot's world transform (R, t).
__device__ __forceinline__ void place_moving(const MovingGeom& g, const float* R, const float* t, float* out) {
  float c[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) c[r] = fmaf(R[6 + r], g.p[2], fmaf(R[3 + r], g.p[1], fmaf(R[r], g.p[0], t[r])));
  if (g.type == G_SPHERE) {
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = g.r;
  } else if (g.type == G_CAPSULE) {
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = g.r;
#pragma unroll
    for (int r = 0; r < 3; ++r) out[4 + r] = fmaf(R[6 + r], g.z[2], fmaf(R[3 + r], g.z[1], R[r] * g.z[0]));
    out[7] = g.hl;
  } else {  // box: axes = columns of R * Rb
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float ax[3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
        ax[r] = fmaf(R[6 + r], g.R[a * 3 + 2], fmaf(R[3 + r], g.R[a * 3 + 1], R[r] * g.R[a * 3]));
      out[4 * a + 0] = ax[0];
      out[4 * a + 1] = ax[1];
      out[4 * a + 2] = ax[2];
      out[4 * a + 3] = -fmaf(ax[2], c[2], fmaf(ax[1], c[1], ax[0] * c[0]));
    }
    out[12] = g.h[0]; out[13] = g.h[1]; out[14] = g.h[2]; out[15] = 0.f;
  }
}

// --------------------------------------------------------------- pair tests
// All return true when the pair COLLIDES.

__device__ __forceinline__ bool sph_sph_hit(const float* a, const float* b) {
  float d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  float dd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
  float rr = a[3] + b[3];
  return !(dd >= rr * rr);
}

// sphere (c, r) vs box in WG format.
__device__ __forceinline__ bool sph_box_hit(const float* c, float r, const float* B) {
  float e2 = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float l = fmaf(B[4 * i + 2], c[2], fmaf(B[4 * i + 1], c[1], fmaf(B[4 * i], c[0], B[4 * i + 3])));
    float e = fmaxf(fabsf(l) - B[12 + i], 0.f);
    e2 = fmaf(e, e, e2);
  }
  return !(e2 >= r * r);
}

// sphere (c, r) vs an axis-aligned box [p 0 | h 0]: the WG test with unit axes,
// which computes exactly c_i - p_i for the box coordinates.
__device__ __forceinline__ bool sph_abox_hit(const float* c, float r, const float4& P, const float4& H) {
  float e0 = fmaxf(fabsf(c[0] - P.x) - H.x, 0.f);
  float e1 = fmaxf(fabsf(c[1] - P.y) - H.y, 0.f);
  float e2 = fmaxf(fabsf(c[2] - P.z) - H.z, 0.f);
  float s = fmaf(e2, e2, fmaf(e1, e1, e0 * e0));
  return !(s >= r * r);
}

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fmaxf(lo, fminf(x, hi)); }

// squared distance of point c to capsule segment (a, u, hl)
__device__ __forceinline__ float pt_seg_d2(const float* c, const float* C) {
  float d0 = c[0] - C[0], d1 = c[1] - C[1], d2 = c[2] - C[2];
  float t = clampf(fmaf(d2, C[6], fmaf(d1, C[5], d0 * C[4])), -C[7], C[7]);
  float e0 = fmaf(-t, C[4], d0), e1 = fmaf(-t, C[5], d1), e2 = fmaf(-t, C[6], d2);
  return fmaf(e2, e2, fmaf(e1, e1, e0 * e0));
}

__device__ __forceinline__ bool sph_cap_hit(const float* S, const float* C) {
  float rr = S[3] + C[3];
  return !(pt_seg_d2(S, C) >= rr * rr);
}

// Squared distance between capsule segments (Ericson 2005, section 5.1.9, in
// centre/half-length form with unit directions).
__device__ __forceinline__ float seg_seg_d2(const float* A, const float* B) {
  float r0 = A[0] - B[0], r1 = A[1] - B[1], r2 = A[2] - B[2];
  float b = fmaf(A[6], B[6], fmaf(A[5], B[5], A[4] * B[4]));
  float c = fmaf(A[6], r2, fmaf(A[5], r1, A[4] * r0));
  float f = fmaf(B[6], r2, fmaf(B[5], r1, B[4] * r0));
  float den = fmaf(-b, b, 1.f);
  float h1 = A[7], h2 = B[7];
  float s = den > 1e-12f ? clampf(fmaf(b, f, -c) / den, -h1, h1) : 0.f;
  float t = fmaf(b, s, f);
  if (t < -h2) {
    t = -h2;
    s = clampf(fmaf(-b, h2, -c), -h1, h1);
  } else if (t > h2) {
    t = h2;
    s = clampf(fmaf(b, h2, -c), -h1, h1);
  }
  float e0 = fmaf(s, A[4], r0) - t * B[4];
  float e1 = fmaf(s, A[5], r1) - t * B[5];
  float e2 = fmaf(s, A[6], r2) - t * B[6];
  return fmaf(e2, e2, fmaf(e1, e1, e0 * e0));
}

// Squared distance between capsule segment C and box B (WG formats): the
// convex piecewise-quadratic f(t) = sum_i max(|l_i + t w_i| - h_i, 0)^2 is
// minimised between the largest breakpoint with f' < 0 and the smallest with
// f' >= 0, where it is a single quadratic.
__device__ __forceinline__ float seg_box_d2(const float* C, const float* B) {
  float l[3], w[3], h[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    l[i] = fmaf(B[4 * i + 2], C[2], fmaf(B[4 * i + 1], C[1], fmaf(B[4 * i], C[0], B[4 * i + 3])));
    w[i] = fmaf(B[4 * i + 2], C[6], fmaf(B[4 * i + 1], C[5], B[4 * i] * C[4]));
    h[i] = B[12 + i];
  }
  const float hl = C[7];
  auto fprime = [&](float t) {
    float g = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float x = fmaf(t, w[i], l[i]);
      float ex = fmaxf(fabsf(x) - h[i], 0.f);
      g = fmaf(copysignf(ex, x), w[i], g);
    }
    return g;
  };
  auto fval = [&](float t) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float x = fmaf(t, w[i], l[i]);
      float ex = fmaxf(fabsf(x) - h[i], 0.f);
      s = fmaf(ex, ex, s);
    }
    return s;
  };
  if (fprime(-hl) >= 0.f) return fval(-hl);
  if (fprime(hl) <= 0.f) return fval(hl);
  float L = -hl, U = hl;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (w[i] == 0.f) continue;
#pragma unroll
    for (int sg = -1; sg <= 1; sg += 2) {
      float c = (sg * h[i] - l[i]) / w[i];
      if (!(c > -hl && c < hl)) continue;
      if (fprime(c) < 0.f)
        L = fmaxf(L, c);
      else
        U = fminf(U, c);
    }
  }
  float m = 0.5f * (L + U);
  float num = 0.f, den = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float x = fmaf(m, w[i], l[i]);
    if (fabsf(x) > h[i]) {
      float sh = copysignf(h[i], x);
      num = fmaf(w[i], l[i] - sh, num);
      den = fmaf(w[i], w[i], den);
    }
  }
  float ts = den > 0.f ? clampf(-num / den, L, U) : L;
  return fval(ts);
}

__device__ __forceinline__ bool cap_box_hit(const float* C, const float* B) {
  return !(seg_box_d2(C, B) >= C[3] * C[3]);
}

__device__ __forceinline__ bool cap_cap_hit(const float* A, const float* B) {
  float rr = A[3] + B[3];
  return !(seg_seg_d2(A, B) >= rr * rr);
}

// Box-box separating-axis test (cuda_geometry_utilities.h:67-125): 15 axes,
// lhs = |(pA - pB) . axis|, rhs = sum of the projected half extents; the
// pair is separated iff lhs > rhs on some axis.
__device__ __forceinline__ bool box_box_hit(const float* A, const float* B) {
  float pa[3], pb[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    pa[r] = -fmaf(A[8 + r], A[11], fmaf(A[4 + r], A[7], A[r] * A[3]));
    pb[r] = -fmaf(B[8 + r], B[11], fmaf(B[4 + r], B[7], B[r] * B[3]));
  }
  float d[3] = {pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]};
  auto sep = [&](float x, float y, float z) {
    float lhs = fabsf(fmaf(d[2], z, fmaf(d[1], y, d[0] * x)));
    float rhs = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      rhs += A[12 + i] * fabsf(fmaf(A[4 * i + 2], z, fmaf(A[4 * i + 1], y, A[4 * i] * x)));
      rhs += B[12 + i] * fabsf(fmaf(B[4 * i + 2], z, fmaf(B[4 * i + 1], y, B[4 * i] * x)));
    }
    return lhs > rhs;
  };
#pragma unroll
  for (int i = 0; i < 3; ++i)
    if (sep(A[4 * i], A[4 * i + 1], A[4 * i + 2]) || sep(B[4 * i], B[4 * i + 1], B[4 * i + 2])) return false;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float* a = A + 4 * i;
      const float* b = B + 4 * j;
      float x = a[1] * b[2] - a[2] * b[1];
      float y = a[2] * b[0] - a[0] * b[2];
      float z = a[0] * b[1] - a[1] * b[0];
      if (sep(x, y, z)) return false;
    }
  return true;
}

// Generic dispatch on types (WG poses).
__device__ __forceinline__ bool pair_hit(int ta, const float* A, int tb, const float* B) {
  if (ta == G_SPHERE && tb == G_SPHERE) return sph_sph_hit(A, B);
  if (ta == G_SPHERE && tb == G_BOX) return sph_box_hit(A, A[3], B);
  if (ta == G_BOX && tb == G_SPHERE) return sph_box_hit(B, B[3], A);
  if (ta == G_SPHERE && tb == G_CAPSULE) return sph_cap_hit(A, B);
  if (ta == G_CAPSULE && tb == G_SPHERE) return sph_cap_hit(B, A);
  if (ta == G_CAPSULE && tb == G_BOX) return cap_box_hit(A, B);
  if (ta == G_BOX && tb == G_CAPSULE) return cap_box_hit(B, A);
  if (ta == G_CAPSULE && tb == G_CAPSULE) return cap_cap_hit(A, B);
  return box_box_hit(A, B);
}

}  // namespace csd
