// csd_oracle.cpp -- CPU oracle for the CSDecomp hot path (TEST INFRASTRUCTURE).
//
// Checker only: loaded by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline / reference arms. Never linked into the product library.
//
// Arithmetic: this file is compiled with -ffp-contract=off so that every
// a*b+c is a rounded multiply followed by a rounded add, as in the
// reference's x86 build of Eigen (no FMA). Where an explicit fmaf() appears it
// restates an operation the build's sampler specifies as fused.
#include "csd_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { FIXED = 0, REVOLUTE = 1, PRISMATIC = 2 };
enum { BOX = 0, SPHERE = 1, CYLINDER = 2, CAPSULE = 3 };

template <typename T>
struct M4 {  // column-major 4x4, m[c*4+r]
  T m[16];
  T& operator()(int r, int c) { return m[c * 4 + r]; }
  T operator()(int r, int c) const { return m[c * 4 + r]; }
};

template <typename T>
M4<T> identity4() {
  M4<T> x;
  for (int i = 0; i < 16; ++i) x.m[i] = T(0);
  x(0, 0) = x(1, 1) = x(2, 2) = x(3, 3) = T(1);
  return x;
}

// Coefficient-wise 4x4 product, k summed in order 0..3 (Eigen's lazy product
// for fixed 4x4 on the CPU path of minimal_kinematic_tree.cpp:50).
template <typename T>
M4<T> mul4(const M4<T>& a, const M4<T>& b) {
  M4<T> r;
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < 4; ++i) {
      T s = a(i, 0) * b(0, c);
      s = s + a(i, 1) * b(1, c);
      s = s + a(i, 2) * b(2, c);
      s = s + a(i, 3) * b(3, c);
      r(i, c) = s;
    }
  return r;
}

template <typename T>
M4<T> load4(const float* src) {
  M4<T> x;
  for (int i = 0; i < 16; ++i) x.m[i] = T(src[i]);
  return x;
}

// Rodrigues' rotation R = c I + (1-c) a a^T + s [a]_x, written out in the
// order of Eigen::AngleAxis::toRotationMatrix used at
// minimal_kinematic_tree.cpp:43-46.
template <typename T>
void rodrigues(T angle, const T* a, M4<T>* X) {
  T s = std::sin(angle), c = std::cos(angle);
  T sa[3] = {s * a[0], s * a[1], s * a[2]};
  T oc = T(1) - c;
  T ca[3] = {oc * a[0], oc * a[1], oc * a[2]};
  T t;
  t = ca[0] * a[1];
  (*X)(0, 1) = t - sa[2];
  (*X)(1, 0) = t + sa[2];
  t = ca[0] * a[2];
  (*X)(0, 2) = t + sa[1];
  (*X)(2, 0) = t - sa[1];
  t = ca[1] * a[2];
  (*X)(1, 2) = t - sa[0];
  (*X)(2, 1) = t + sa[0];
  (*X)(0, 0) = ca[0] * a[0] + c;
  (*X)(1, 1) = ca[1] * a[1] + c;
  (*X)(2, 2) = ca[2] * a[2] + c;
}

// FK for one configuration: computeLinkFrameToWorldTransformsMinimal,
// csdecomp/src/plant/minimal_kinematic_tree.cpp:10-58.
template <typename T>
void fk_one(const orc_plant_t* p, const float* q, M4<T>* tf) {
  tf[0] = identity4<T>();
  for (int t = 0; t < p->num_joints; ++t) {
    int j = p->joint_traversal_sequence[t];
    int pl = p->joint_parent_link[j], cl = p->joint_child_link[j];
    M4<T> X_PL_J = load4<T>(p->joint_X_PL_J + 16 * j);
    T qv = T(0);
    int type = p->joint_type[j];
    if (type != FIXED) qv = T(q[p->joint_idx_to_config_idx[j]]);
    M4<T> X_J_L = identity4<T>();
    T ax[3] = {T(p->joint_axis[3 * j]), T(p->joint_axis[3 * j + 1]), T(p->joint_axis[3 * j + 2])};
    if (type == REVOLUTE) {
      rodrigues<T>(qv, ax, &X_J_L);
    } else if (type == PRISMATIC) {
      X_J_L(0, 3) = T(0) + ax[0] * qv;
      X_J_L(1, 3) = T(0) + ax[1] * qv;
      X_J_L(2, 3) = T(0) + ax[2] * qv;
    }
    tf[cl] = mul4(mul4(tf[pl], X_PL_J), X_J_L);
  }
}

// ---------------------------------------------------------------- geometry
template <typename T>
struct Pose {
  T p[3];
  T R[9];  // column-major 3x3
};

template <typename T>
Pose<T> pose_of(const M4<T>& X) {
  Pose<T> o;
  for (int i = 0; i < 3; ++i) o.p[i] = X(i, 3);
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o.R[c * 3 + r] = X(r, c);
  return o;
}

template <typename T>
T dot3(const T* a, const T* b) {
  T s = a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}

// sphere-sphere: GPU rule cuda_geometry_utilities.h:16-20 (d^2 >= (ra+rb)^2),
// CPU rule collision_checker.cpp:110-115 (|d| > ra+rb).
bool sphere_sphere_free(float ra, const float* pa, float rb, const float* pb, int rule) {
  float d[3] = {pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]};
  float d2 = dot3(d, d);
  if (rule == ORC_RULE_GPU) return d2 >= (ra + rb) * (ra + rb);
  return std::sqrt(d2) > ra + rb;
}

// sphere-box: cuda_geometry_utilities.h:31-55 / collision_checker.cpp:172-199.
bool sphere_box_free(float r, const float* c, const float* dims, const Pose<float>& box, int rule) {
  float h[3] = {dims[0] * 0.5f, dims[1] * 0.5f, dims[2] * 0.5f};
  float d[3] = {c[0] - box.p[0], c[1] - box.p[1], c[2] - box.p[2]};
  float l[3];
  for (int i = 0; i < 3; ++i) l[i] = dot3(box.R + 3 * i, d);  // R^T d
  float e[3];
  for (int i = 0; i < 3; ++i) {
    float cl = std::max(-h[i], std::min(l[i], h[i]));
    e[i] = cl - l[i];
  }
  float d2 = dot3(e, e);
  if (rule == ORC_RULE_GPU) return d2 >= r * r;
  return d2 > r * r;
}

void cross3(const float* a, const float* b, float* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// box-box SAT over 15 axes, lhs/rhs accumulated in double:
// cuda_geometry_utilities.h:67-125, collision_checker.cpp:127-180 (CPU adds a
// bounding-distance prefilter that never changes the verdict).
bool box_box_free(const float* da, const Pose<float>& A, const float* db, const Pose<float>& B,
                  int rule) {
  if (rule == ORC_RULE_CPU) {
    float maxlen = std::max(std::max(std::max(da[0], da[1]), da[2]),
                            std::max(std::max(db[0], db[1]), db[2]));
    float d[3] = {A.p[0] - B.p[0], A.p[1] - B.p[1], A.p[2] - B.p[2]};
    if (std::sqrt(dot3(d, d)) > 2.0f * std::sqrt(3.0f) * maxlen) return true;
  }
  const float* a[3] = {A.R, A.R + 3, A.R + 6};
  const float* b[3] = {B.R, B.R + 3, B.R + 6};
  float axes[15][3];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) {
      axes[i][k] = a[i][k];
      axes[3 + i][k] = b[i][k];
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) cross3(a[i], b[j], axes[6 + 3 * i + j]);
  float pab[3] = {A.p[0] - B.p[0], A.p[1] - B.p[1], A.p[2] - B.p[2]};
  for (int s = 0; s < 15; ++s) {
    const float* ax = axes[s];
    double lhs = std::fabs(dot3(pab, ax));
    double rhs = std::fabs((da[0] / 2) * dot3(a[0], ax));
    rhs = rhs + std::fabs((da[1] / 2) * dot3(a[1], ax));
    rhs = rhs + std::fabs((da[2] / 2) * dot3(a[2], ax));
    rhs = rhs + std::fabs((db[0] / 2) * dot3(b[0], ax));
    rhs = rhs + std::fabs((db[1] / 2) * dot3(b[1], ax));
    rhs = rhs + std::fabs((db[2] / 2) * dot3(b[2], ax));
    if (lhs > rhs) return true;
  }
  return false;
}

// ---- capsules (no reference semantics): sphere-swept segment along local z.
template <typename T>
T clampT(T x, T lo, T hi) {
  return std::max(lo, std::min(x, hi));
}

template <typename T>
void capsule_segment(const Pose<T>& P, T length, T* a, T* u, T* hl) {
  for (int i = 0; i < 3; ++i) {
    a[i] = P.p[i];
    u[i] = P.R[6 + i];
  }
  *hl = length * T(0.5);
}

// Squared distance point c -> segment a + t u, |t| <= hl (u unit).
template <typename T>
T point_segment_d2(const T* c, const T* a, const T* u, T hl) {
  T d[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  T t = clampT(dot3(d, u), -hl, hl);
  T e[3] = {d[0] - t * u[0], d[1] - t * u[1], d[2] - t * u[2]};
  return dot3(e, e);
}

// Squared distance between segments a1+s u1 (|s|<=h1) and a2+t u2 (|t|<=h2),
// u1,u2 unit: the clamped closest-point solution of Ericson, "Real-Time
// Collision Detection" (2005), section 5.1.9, in centre/half-length form.
template <typename T>
T segment_segment_d2(const T* a1, const T* u1, T h1, const T* a2, const T* u2, T h2) {
  T r[3] = {a1[0] - a2[0], a1[1] - a2[1], a1[2] - a2[2]};
  T b = dot3(u1, u2);
  T c = dot3(u1, r);
  T f = dot3(u2, r);
  T den = T(1) - b * b;
  T s;
  if (den > T(1e-12)) {
    s = clampT((b * f - c) / den, -h1, h1);
  } else {
    s = T(0);
  }
  T t = b * s + f;
  if (t < -h2) {
    t = -h2;
    s = clampT(-b * h2 - c, -h1, h1);
  } else if (t > h2) {
    t = h2;
    s = clampT(b * h2 - c, -h1, h1);
  }
  T e[3];
  for (int i = 0; i < 3; ++i) e[i] = (a1[i] + s * u1[i]) - (a2[i] + t * u2[i]);
  return dot3(e, e);
}

// Squared distance between segment a + t u (|t| <= hl) and an oriented box.
// f(t) = sum_i max(|l_i + t w_i| - h_i, 0)^2 is convex and piecewise
// quadratic; its minimiser lies between the largest breakpoint with f' < 0
// and the smallest with f' >= 0, where f is a single quadratic.
template <typename T>
T segment_box_d2(const T* a, const T* u, T hl, const T* dims, const Pose<T>& B) {
  T h[3] = {dims[0] * T(0.5), dims[1] * T(0.5), dims[2] * T(0.5)};
  T d[3] = {a[0] - B.p[0], a[1] - B.p[1], a[2] - B.p[2]};
  T l[3], w[3];
  for (int i = 0; i < 3; ++i) {
    l[i] = dot3(B.R + 3 * i, d);
    w[i] = dot3(B.R + 3 * i, u);
  }
  auto fprime = [&](T t) {
    T g = T(0);
    for (int i = 0; i < 3; ++i) {
      T x = l[i] + t * w[i];
      T ex = std::max(std::fabs(x) - h[i], T(0));
      g = g + (x >= T(0) ? ex : -ex) * w[i];
    }
    return g;
  };
  auto fval = [&](T t) {
    T s = T(0);
    for (int i = 0; i < 3; ++i) {
      T x = l[i] + t * w[i];
      T ex = std::max(std::fabs(x) - h[i], T(0));
      s = s + ex * ex;
    }
    return s;
  };
  T lo = -hl, hi = hl;
  if (fprime(lo) >= T(0)) return fval(lo);
  if (fprime(hi) <= T(0)) return fval(hi);
  T L = lo, U = hi;
  for (int i = 0; i < 3; ++i) {
    if (w[i] == T(0)) continue;
    for (int sgn = -1; sgn <= 1; sgn += 2) {
      T c = (T(sgn) * h[i] - l[i]) / w[i];
      if (!(c > lo && c < hi)) continue;
      if (fprime(c) < T(0))
        L = std::max(L, c);
      else
        U = std::min(U, c);
    }
  }
  T m = T(0.5) * (L + U);
  T num = T(0), den = T(0);
  for (int i = 0; i < 3; ++i) {
    T x = l[i] + m * w[i];
    if (std::fabs(x) > h[i]) {
      T sh = x >= T(0) ? h[i] : -h[i];
      num = num + w[i] * (l[i] - sh);
      den = den + w[i] * w[i];
    }
  }
  T ts = den > T(0) ? clampT(-num / den, L, U) : L;
  return fval(ts);
}

// Generic pair test on world poses. Returns 1 free, 0 colliding, -1 unsupported.
int pair_free_posed(int ta, const float* da, const Pose<float>& A, int tb, const float* db,
                    const Pose<float>& B, int rule) {
  if (ta == CYLINDER || tb == CYLINDER) return -1;
  if (ta == SPHERE && tb == SPHERE) return sphere_sphere_free(da[0], A.p, db[0], B.p, rule);
  if (ta == SPHERE && tb == BOX) return sphere_box_free(da[0], A.p, db, B, rule);
  if (ta == BOX && tb == SPHERE) return sphere_box_free(db[0], B.p, da, A, rule);
  if (ta == BOX && tb == BOX) return box_box_free(da, A, db, B, rule);
  // capsule cases
  auto cmp = [rule](float d2, float r) { return rule == ORC_RULE_GPU ? d2 >= r * r : d2 > r * r; };
  if (ta == CAPSULE || tb == CAPSULE) {
    bool swap = ta != CAPSULE;
    int tc = swap ? tb : ta, to = swap ? ta : tb;
    (void)tc;
    const float* dc = swap ? db : da;
    const float* dn = swap ? da : db;
    const Pose<float>& C = swap ? B : A;
    const Pose<float>& O = swap ? A : B;
    float a[3], u[3], hl;
    capsule_segment<float>(C, dc[1], a, u, &hl);
    if (to == SPHERE) return cmp(point_segment_d2<float>(O.p, a, u, hl), dc[0] + dn[0]);
    if (to == BOX) return cmp(segment_box_d2<float>(a, u, hl, dn, O), dc[0]);
    float a2[3], u2[3], hl2;
    capsule_segment<float>(O, dn[1], a2, u2, &hl2);
    return cmp(segment_segment_d2<float>(a, u, hl, a2, u2, hl2), dc[0] + dn[0]);
  }
  return -1;
}

// FP64 signed distance of a pair (for the contact band classification).
double pair_sd64(int ta, const float* dA, const Pose<double>& A, int tb, const float* dB,
                 const Pose<double>& B) {
  double da[3] = {dA[0], dA[1], dA[2]}, db[3] = {dB[0], dB[1], dB[2]};
  auto sph_box = [](double r, const double* c, const double* dims, const Pose<double>& X) {
    double d[3] = {c[0] - X.p[0], c[1] - X.p[1], c[2] - X.p[2]};
    double e2 = 0, depth = 1e300;
    for (int i = 0; i < 3; ++i) {
      double l = dot3(X.R + 3 * i, d);
      double h = dims[i] * 0.5;
      double ex = std::max(std::fabs(l) - h, 0.0);
      e2 += ex * ex;
      depth = std::min(depth, h - std::fabs(l));
    }
    if (e2 > 0) return std::sqrt(e2) - r;
    return -r - std::max(depth, 0.0);
  };
  if (ta == SPHERE && tb == SPHERE) {
    double d[3] = {A.p[0] - B.p[0], A.p[1] - B.p[1], A.p[2] - B.p[2]};
    return std::sqrt(dot3(d, d)) - da[0] - db[0];
  }
  if (ta == SPHERE && tb == BOX) return sph_box(da[0], A.p, db, B);
  if (ta == BOX && tb == SPHERE) return sph_box(db[0], B.p, da, A);
  if (ta == BOX && tb == BOX) {
    const double* a[3] = {A.R, A.R + 3, A.R + 6};
    const double* b[3] = {B.R, B.R + 3, B.R + 6};
    double axes[15][3];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) {
        axes[i][k] = a[i][k];
        axes[3 + i][k] = b[i][k];
      }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double* o = axes[6 + 3 * i + j];
        o[0] = a[i][1] * b[j][2] - a[i][2] * b[j][1];
        o[1] = a[i][2] * b[j][0] - a[i][0] * b[j][2];
        o[2] = a[i][0] * b[j][1] - a[i][1] * b[j][0];
      }
    double pab[3] = {A.p[0] - B.p[0], A.p[1] - B.p[1], A.p[2] - B.p[2]};
    double best = -1e300;
    for (int s = 0; s < 15; ++s) {
      const double* ax = axes[s];
      double n = std::sqrt(dot3(ax, ax));
      if (n < 1e-9) continue;
      double lhs = std::fabs(dot3(pab, ax));
      double rhs = 0;
      for (int i = 0; i < 3; ++i) rhs += std::fabs(da[i] * 0.5 * dot3(a[i], ax));
      for (int i = 0; i < 3; ++i) rhs += std::fabs(db[i] * 0.5 * dot3(b[i], ax));
      best = std::max(best, (lhs - rhs) / n);
    }
    return best;
  }
  bool swap = ta != CAPSULE;
  int to = swap ? ta : tb;
  const double* dc = swap ? db : da;
  const double* dn = swap ? da : db;
  const Pose<double>& C = swap ? B : A;
  const Pose<double>& O = swap ? A : B;
  double a[3], u[3], hl;
  capsule_segment<double>(C, dc[1], a, u, &hl);
  if (to == SPHERE) return std::sqrt(point_segment_d2<double>(O.p, a, u, hl)) - dc[0] - dn[0];
  if (to == BOX) return std::sqrt(segment_box_d2<double>(a, u, hl, dn, O)) - dc[0];
  double a2[3], u2[3], hl2;
  capsule_segment<double>(O, dn[1], a2, u2, &hl2);
  return std::sqrt(segment_segment_d2<double>(a, u, hl, a2, u2, hl2)) - dc[0] - dn[0];
}

struct Workspace {
  std::vector<M4<float>> tf;
  std::vector<M4<double>> tf64;
};

// Point check for one config: checkCollisionFree / checkCollisionFreeVoxels,
// collision_checker.cpp:9-39 and 55-89 (without the per-pair stdout print;
// the verdict does not depend on pair order, so the loop returns at the first
// collision as checkCollisionFreeVoxels does).
bool check_one(const orc_plant_t* p, const float* q, int rule, const float* vox, int nv, float vr,
               const int32_t* rids, int nr, Workspace& ws) {
  ws.tf.resize(p->num_links);
  fk_one<float>(p, q, ws.tf.data());
  for (int k = 0; k < p->num_collision_pairs; ++k) {
    int ia = p->collision_pairs_flat[2 * k], ib = p->collision_pairs_flat[2 * k + 1];
    M4<float> XA = mul4(ws.tf[p->geom_link_index[ia]], load4<float>(p->geom_X_L_B + 16 * ia));
    M4<float> XB = mul4(ws.tf[p->geom_link_index[ib]], load4<float>(p->geom_X_L_B + 16 * ib));
    int r = pair_free_posed(p->geom_type[ia], p->geom_dimensions + 3 * ia, pose_of(XA),
                            p->geom_type[ib], p->geom_dimensions + 3 * ib, pose_of(XB), rule);
    if (r != 1) return false;
  }
  if (nv > 0) {
    for (int g = 0; g < nr; ++g) {
      int ig = rids[g];
      M4<float> X = mul4(ws.tf[p->geom_link_index[ig]], load4<float>(p->geom_X_L_B + 16 * ig));
      Pose<float> P = pose_of(X);
      float vd[3] = {vr, -1.f, -1.f};
      for (int v = 0; v < nv; ++v) {
        Pose<float> V;
        for (int i = 0; i < 3; ++i) V.p[i] = vox[3 * v + i];
        for (int i = 0; i < 9; ++i) V.R[i] = (i % 4 == 0) ? 1.f : 0.f;
        if (pair_free_posed(SPHERE, vd, V, p->geom_type[ig], p->geom_dimensions + 3 * ig, P, rule) != 1)
          return false;
      }
    }
  }
  return true;
}

void sd_one(const orc_plant_t* p, const float* q, const float* vox, int nv, float vr,
            const int32_t* rids, int nr, Workspace& ws, uint8_t* verdict, double* min_sd) {
  ws.tf64.resize(p->num_links);
  fk_one<double>(p, q, ws.tf64.data());
  bool free = true;
  double mabs = 1e300;
  for (int k = 0; k < p->num_collision_pairs; ++k) {
    int ia = p->collision_pairs_flat[2 * k], ib = p->collision_pairs_flat[2 * k + 1];
    M4<double> XA = mul4(ws.tf64[p->geom_link_index[ia]], load4<double>(p->geom_X_L_B + 16 * ia));
    M4<double> XB = mul4(ws.tf64[p->geom_link_index[ib]], load4<double>(p->geom_X_L_B + 16 * ib));
    double sd = pair_sd64(p->geom_type[ia], p->geom_dimensions + 3 * ia, pose_of(XA),
                          p->geom_type[ib], p->geom_dimensions + 3 * ib, pose_of(XB));
    if (sd <= 0) free = false;
    mabs = std::min(mabs, sd);
  }
  for (int g = 0; g < nr && nv > 0; ++g) {
    int ig = rids[g];
    M4<double> X = mul4(ws.tf64[p->geom_link_index[ig]], load4<double>(p->geom_X_L_B + 16 * ig));
    Pose<double> P = pose_of(X);
    float vd[3] = {vr, -1.f, -1.f};
    for (int v = 0; v < nv; ++v) {
      Pose<double> V;
      for (int i = 0; i < 3; ++i) V.p[i] = vox[3 * v + i];
      for (int i = 0; i < 9; ++i) V.R[i] = (i % 4 == 0) ? 1.0 : 0.0;
      double sd = pair_sd64(SPHERE, vd, V, p->geom_type[ig], p->geom_dimensions + 3 * ig, P);
      if (sd <= 0) free = false;
      mabs = std::min(mabs, sd);
    }
  }
  *verdict = free ? 1 : 0;
  *min_sd = mabs;
}

int validate(const orc_plant_t* p) {
  for (int g = 0; g < p->num_geometries; ++g)
    if (p->geom_type[g] == CYLINDER || p->geom_type[g] < 0 || p->geom_type[g] > CAPSULE) return -1;
  for (int k = 0; k < 2 * p->num_collision_pairs; ++k)
    if (p->collision_pairs_flat[k] < 0 || p->collision_pairs_flat[k] >= p->num_geometries) return -2;
  return 0;
}

// ------------------------------------------------------------------ edges
float norm_l2(const float* a, const float* b, int d) {
  float s = 0.f;
  for (int i = 0; i < d; ++i) {
    float x = b[i] - a[i];
    s = s + x * x;
  }
  return std::sqrt(s);
}

float norm_linf(const float* a, const float* b, int d) {
  float m = 0.f;
  for (int i = 0; i < d; ++i) m = std::max(m, std::fabs(b[i] - a[i]));
  return m;
}

void lerp(const float* q1, const float* q2, int d, float t, float* out) {
  float omt = 1.0f - t;
  for (int i = 0; i < d; ++i) out[i] = t * q2[i] + omt * q1[i];
}

}  // namespace

// ======================================================================
extern "C" {

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static void set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_fk_f32(const orc_plant_t* p, const float* q, int64_t n, float* tf) {
  std::vector<M4<float>> buf(p->num_links);
  for (int64_t i = 0; i < n; ++i) {
    fk_one<float>(p, q + i * p->num_configuration_variables, buf.data());
    std::memcpy(tf + i * 16 * p->num_links, buf.data(), sizeof(float) * 16 * p->num_links);
  }
  return 0;
}

int orc_fk_f64(const orc_plant_t* p, const float* q, int64_t n, double* tf) {
  std::vector<M4<double>> buf(p->num_links);
  for (int64_t i = 0; i < n; ++i) {
    fk_one<double>(p, q + i * p->num_configuration_variables, buf.data());
    std::memcpy(tf + i * 16 * p->num_links, buf.data(), sizeof(double) * 16 * p->num_links);
  }
  return 0;
}

int orc_check_points(const orc_plant_t* p, const float* q, int64_t n, int rule, const float* voxels,
                     int32_t nv, float vr, const int32_t* rids, int32_t nr, uint8_t* out,
                     int nthreads) {
  if (validate(p)) return -1;
  set_threads(nthreads);
  const int d = p->num_configuration_variables;
#pragma omp parallel
  {
    Workspace ws;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i)
      out[i] = check_one(p, q + i * d, rule, voxels, nv, vr, rids, nr, ws) ? 1 : 0;
  }
  return 0;
}

int orc_signed_distance_f64(const orc_plant_t* p, const float* q, int64_t n, const float* voxels,
                            int32_t nv, float vr, const int32_t* rids, int32_t nr,
                            uint8_t* verdict64, double* min_abs_sd, int nthreads) {
  if (validate(p)) return -1;
  set_threads(nthreads);
  const int d = p->num_configuration_variables;
#pragma omp parallel
  {
    Workspace ws;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i)
      sd_one(p, q + i * d, voxels, nv, vr, rids, nr, ws, verdict64 + i, min_abs_sd + i);
  }
  return 0;
}

int64_t orc_edge_num_points(const float* q1, const float* q2, int32_t d, float step, int mode) {
  if (mode == ORC_EDGE_L2_REF) {
    // collision_checker.cpp:44: t_steps = ceil(norm / step); k = 0..t_steps-1
    return (int64_t)std::ceil(norm_l2(q1, q2, d) / step);
  }
  if (mode == ORC_EDGE_LINF) {
    int64_t T = (int64_t)std::ceil(norm_linf(q1, q2, d) / step);
    return T + 1;
  }
  // cuda_visibility_graph.cu:69: n = dist / step + 2 (float, truncated)
  float x = norm_l2(q1, q2, d) / step + 2.0f;
  return (int64_t)(uint32_t)x;
}

void orc_edge_point(const float* q1, const float* q2, int32_t d, float step, int mode, int64_t k,
                    float* out) {
  if (mode == ORC_EDGE_L2_REF) {
    int64_t T = orc_edge_num_points(q1, q2, d, step, mode);
    float t = (float)(k / (1.0 * T));  // collision_checker.cpp:46
    lerp(q1, q2, d, t, out);
    return;
  }
  if (mode == ORC_EDGE_LINF) {
    int64_t T = orc_edge_num_points(q1, q2, d, step, mode) - 1;
    if (T == 0) {
      std::memcpy(out, q1, sizeof(float) * d);
      return;
    }
    float t = (float)(k / (1.0 * T));
    lerp(q1, q2, d, t, out);
    return;
  }
  // VG ordering: start, end, then interior points (cuda_visibility_graph.cu:152-170)
  int64_t n = orc_edge_num_points(q1, q2, d, step, mode);
  if (k == 0) {
    std::memcpy(out, q1, sizeof(float) * d);
    return;
  }
  if (k == 1) {
    std::memcpy(out, q2, sizeof(float) * d);
    return;
  }
  float t_step = (float)(1.0 / (double)(n - 1));
  float t = t_step * (float)(k - 1);
  lerp(q1, q2, d, t, out);
}

int orc_check_edges(const orc_plant_t* p, const float* starts, const float* ends, int64_t e,
                    float step, int mode, int rule, uint8_t* out, int64_t* points_checked,
                    int nthreads) {
  if (validate(p)) return -1;
  set_threads(nthreads);
  const int d = p->num_configuration_variables;
#pragma omp parallel
  {
    Workspace ws;
    std::vector<float> qk(d);
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < e; ++i) {
      const float* q1 = starts + i * d;
      const float* q2 = ends + i * d;
      int64_t n = orc_edge_num_points(q1, q2, d, step, mode);
      uint8_t free = 1;
      int64_t k = 0;
      for (; k < n; ++k) {
        orc_edge_point(q1, q2, d, step, mode, k, qk.data());
        if (!check_one(p, qk.data(), rule, nullptr, 0, 0.f, nullptr, 0, ws)) {
          free = 0;
          ++k;
          break;
        }
      }
      out[i] = free;
      if (points_checked) points_checked[i] = k;
    }
  }
  return 0;
}

int orc_pair_collision_free(int32_t ta, const float* da, const float* XLBa, const float* XWLa,
                            int32_t tb, const float* db, const float* XLBb, const float* XWLb,
                            int rule) {
  M4<float> XA = mul4(load4<float>(XWLa), load4<float>(XLBa));
  M4<float> XB = mul4(load4<float>(XWLb), load4<float>(XLBb));
  return pair_free_posed(ta, da, pose_of(XA), tb, db, pose_of(XB), rule);
}

}  // extern "C"

// ======================================================================
// Sampler. The reference draws directions with cuRAND's XORWOW stream
// (cuda_hit_and_run_sampling.cu:26,78,107); the build specifies its own
// counter-based stream instead so GPU and CPU draw identical numbers:
//   * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
//     as easy as 1, 2, 3", SC'11), key = (seed lo, seed hi),
//     counter = (step, chain, stream, block);
//   * uniform in (0,1]: ((x >> 8) + 1) * 2^-24; angle fraction in [0,1): (x >> 8) * 2^-24;
//   * Gaussian pairs by Box-Muller with the build's own ln() (atanh series)
//     and sin/cos (Taylor series) written with correctly rounded operations.
namespace {

inline uint32_t mulhi32(uint32_t a, uint32_t b, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *lo = (uint32_t)p;
  return (uint32_t)(p >> 32);
}

void philox4x32_10(const uint32_t in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t lo0, lo1;
    uint32_t hi0 = mulhi32(0xD2511F53u, c0, &lo0);
    uint32_t hi1 = mulhi32(0xCD9E8D57u, c2, &lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

inline float u01_open0(uint32_t x) { return (float)((x >> 8) + 1u) * 5.9604644775390625e-08f; }
inline float u01_open1(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

// ln(u), u in (0,1]: u = m 2^e, m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
// s = (m-1)/(m+1), atanh(s) = s (1 + s^2/3 + s^4/5 + s^6/7 + s^8/9 + s^10/11).
// ln 2 split into a 16-bit head (exact products with e) and a tail.
inline float csd_log_unit(float u) {
  uint32_t bits;
  std::memcpy(&bits, &u, 4);
  int e = (int)(bits >> 23) - 127;
  uint32_t mb = (bits & 0x007fffffu) | 0x3f800000u;
  float m;
  std::memcpy(&m, &mb, 4);
  if (m > 1.41421353816986083984375f) {
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = std::fmaf(s2, 0.0909090936183929443359375f, 0.111111111938953399658203125f);
  p = std::fmaf(s2, p, 0.142857149243354797363281250f);
  p = std::fmaf(s2, p, 0.20000000298023223876953125f);
  p = std::fmaf(s2, p, 0.3333333432674407958984375f);
  p = std::fmaf(s2, p, 1.0f);
  float t = s * p;
  float lnm = t + t;
  float fe = (float)e;
  float lo = std::fmaf(fe, 1.428606765330187045037746429443359375e-06f, lnm);
  return std::fmaf(fe, 0.693145751953125f, lo);
}

// (sin, cos) of 2*pi*v for v in [0,1): quadrant from 4v, x = f*pi/2 with
// f in [0,1), Taylor series through x^13 (sin) and x^14 (cos).
inline void csd_sincos_2pi(float v, float* sn, float* cs) {
  float w = v * 4.0f;
  int qd = (int)w;
  float f = w - (float)qd;
  float x = f * 1.57079637050628662109375f;
  float x2 = x * x;
  float ps = std::fmaf(x2, 1.6059043836821614e-10f, -2.5052108385441720e-08f);
  ps = std::fmaf(x2, ps, 2.7557319223985893e-06f);
  ps = std::fmaf(x2, ps, -1.9841269841269841e-04f);
  ps = std::fmaf(x2, ps, 8.3333333333333333e-03f);
  ps = std::fmaf(x2, ps, -1.6666666666666667e-01f);
  ps = std::fmaf(x2, ps, 1.0f);
  float s = x * ps;
  float pc = std::fmaf(x2, -1.1470745597729725e-11f, 2.0876756987868099e-09f);
  pc = std::fmaf(x2, pc, -2.7557319223985891e-07f);
  pc = std::fmaf(x2, pc, 2.4801587301587302e-05f);
  pc = std::fmaf(x2, pc, -1.3888888888888889e-03f);
  pc = std::fmaf(x2, pc, 4.1666666666666667e-02f);
  pc = std::fmaf(x2, pc, -0.5f);
  float c = std::fmaf(x2, pc, 1.0f);
  switch (qd & 3) {
    case 0: *sn = s; *cs = c; break;
    case 1: *sn = c; *cs = -s; break;
    case 2: *sn = -s; *cs = -c; break;
    default: *sn = -c; *cs = s; break;
  }
}

// Random words for (chain, stream, step): word w comes from Philox block w/4.
struct StepRng {
  uint32_t w[20];
  StepRng(uint64_t seed, uint32_t chain, uint32_t stream, uint32_t step, int nblocks) {
    for (int bl = 0; bl < nblocks; ++bl) {
      uint32_t ctr[4] = {step, chain, stream, (uint32_t)bl};
      philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), w + 4 * bl);
    }
  }
};

// Direction (dim Gaussians) and the theta uniform for one mixing step.
// Gaussian pair g uses words 2g (radius) and 2g+1 (angle); the theta uniform
// is word 2*ceil(dim/2).
void step_draws(uint64_t seed, uint32_t chain, uint32_t stream, uint32_t step, int dim, float* dir,
                float* u_theta) {
  int npairs = (dim + 1) / 2;
  int nwords = 2 * npairs + 1;
  StepRng r(seed, chain, stream, step, (nwords + 3) / 4);
  for (int g = 0; g < npairs; ++g) {
    float u = u01_open0(r.w[2 * g]);
    float v = u01_open1(r.w[2 * g + 1]);
    float rad = std::sqrt(-2.0f * csd_log_unit(u));
    float sn, cs;
    csd_sincos_2pi(v, &sn, &cs);
    dir[2 * g] = rad * cs;
    if (2 * g + 1 < dim) dir[2 * g + 1] = rad * sn;
  }
  *u_theta = u01_open0(r.w[2 * npairs]);
}

// One hit-and-run chain: uniformSampleInHPolyhedronKernel,
// cuda_hit_and_run_sampling.cu:57-118, with dot products accumulated by fmaf
// in index order and theta drawn as in :106-107 (0.999999 scales theta_max only).
bool run_chain(const float* A, const float* b, int F, int d, const float* x0, int mixing,
               uint64_t seed, uint32_t chain, uint32_t stream, float* x) {
  for (int i = 0; i < d; ++i) x[i] = x0[i];
  float dir[16];
  for (int s = 0; s < mixing; ++s) {
    float ut;
    step_draws(seed, chain, stream, (uint32_t)s, d, dir, &ut);
    float tmax = FLT_MAX, tmin = -FLT_MAX;
    for (int f = 0; f < F; ++f) {
      const float* a = A + (int64_t)f * d;
      float ax = a[0] * x[0];
      float ad = a[0] * dir[0];
      for (int k = 1; k < d; ++k) {
        ax = std::fmaf(a[k], x[k], ax);
        ad = std::fmaf(a[k], dir[k], ad);
      }
      float lb = b[f] - ax;
      if (ad < 0.0f)
        tmin = std::max(tmin, lb / ad);
      else if (ad > 0.0f)
        tmax = std::min(tmax, lb / ad);
    }
    if (std::isinf(tmax) || std::isinf(tmin) || tmax < tmin) return false;
    float theta = (float)((double)ut * (0.999999 * (double)tmax - (double)tmin) + (double)tmin);
    for (int k = 0; k < d; ++k) x[k] = std::fmaf(theta, dir[k], x[k]);
  }
  return true;
}

// One EI-ZO chain with carried slacks (the GPU's EI-ZO sampler,
// csdecomp_b200/csrc/sampler_core.cuh run_chain_pairs): the start slacks
// s_f = b_f - a_f . x0 (product of coordinate 0, fmaf in coordinate order,
// then b minus that); per step one dot product a_f . dir per face (same
// order), the theta bounds of cuda_hit_and_run_sampling.cu:83-104 from
// s_f / (a_f . dir), theta as in :106-107, then x_k = fmaf(theta, dir_k, x_k)
// and s_f = fmaf(-theta, a_f . dir, s_f). The reference recomputes b - A x
// every step instead; the draws, the bounds and theta are its. s and ad are
// F floats of scratch.
bool run_chain_carried(const float* A, const float* b, int F, int d, const float* x0, int mixing, uint64_t seed,
                       uint32_t chain, uint32_t stream, float* x, float* s, float* ad) {
  for (int i = 0; i < d; ++i) x[i] = x0[i];
  for (int f = 0; f < F; ++f) {
    const float* a = A + (int64_t)f * d;
    float ax = a[0] * x0[0];
    for (int k = 1; k < d; ++k) ax = std::fmaf(a[k], x0[k], ax);
    s[f] = b[f] - ax;
  }
  float dir[16];
  for (int st = 0; st < mixing; ++st) {
    float ut;
    step_draws(seed, chain, stream, (uint32_t)st, d, dir, &ut);
    float tmax = FLT_MAX, tmin = -FLT_MAX;
    for (int f = 0; f < F; ++f) {
      const float* a = A + (int64_t)f * d;
      float v = a[0] * dir[0];
      for (int k = 1; k < d; ++k) v = std::fmaf(a[k], dir[k], v);
      ad[f] = v;
      if (v < 0.0f)
        tmin = std::max(tmin, s[f] / v);
      else if (v > 0.0f)
        tmax = std::min(tmax, s[f] / v);
    }
    if (std::isinf(tmax) || std::isinf(tmin) || tmax < tmin) return false;
    float theta = (float)((double)ut * (0.999999 * (double)tmax - (double)tmin) + (double)tmin);
    for (int k = 0; k < d; ++k) x[k] = std::fmaf(theta, dir[k], x[k]);
    for (int f = 0; f < F; ++f) s[f] = std::fmaf(-theta, ad[f], s[f]);
  }
  return true;
}

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  philox4x32_10(ctr, key[0], key[1], out);
}

void orc_rng_uniform(uint64_t seed, uint32_t chain, uint32_t stream, uint32_t step, float* out4) {
  StepRng r(seed, chain, stream, step, 1);
  for (int i = 0; i < 4; ++i) out4[i] = u01_open0(r.w[i]);
}

void orc_rng_direction(uint64_t seed, uint32_t chain, uint32_t stream, uint32_t step, int32_t dim,
                       float* dir) {
  float ut;
  step_draws(seed, chain, stream, step, dim, dir, &ut);
  dir[dim] = ut;
}

int orc_hit_and_run(const float* A, const float* b, int32_t F, int32_t d, const float* x0,
                    int32_t S, int32_t mixing, uint64_t seed, uint32_t stream, float* samples,
                    int32_t* num_failed, int nthreads) {
  if (d > 16 || d <= 0) return -1;
  set_threads(nthreads);
  int failed = 0;
#pragma omp parallel for schedule(static) reduction(+ : failed)
  for (int s = 0; s < S; ++s) {
    float x[16];
    bool ok = run_chain(A, b, F, d, x0, mixing, seed, (uint32_t)s, stream, x);
    for (int k = 0; k < d; ++k) samples[(int64_t)s * d + k] = ok ? x[k] : NAN;
    failed += ok ? 0 : 1;
  }
  if (num_failed) *num_failed = failed;
  return 0;
}

uint32_t orc_num_samples_unadaptive(float epsilon, float delta, float tau) {
  // cuda_set_builder_utils.h:198-203 (float arithmetic throughout)
  float one_over = 1.0f / delta;
  float lg = std::log(one_over);
  float num = 2.0f * lg;
  float den = epsilon * tau * tau;
  return (uint32_t)std::ceil(num / den);
}

// EI-ZO: executeEizo, cuda_edge_inflation_zero_order.cu:109-338, with the
// collision compaction of cuda_set_builder_utils.cu:168-186 made
// deterministic (first colliding samples in index order) and the sampler's
// slacks carried from step to step (run_chain_carried).
int orc_eizo(const orc_plant_t* p, const float* ls, const float* le, const float* voxels,
             int32_t nv, float vr, const int32_t* rids, int32_t nr, const orc_eizo_options_t* o,
             float* A, float* b, int32_t* num_faces, int32_t capacity, orc_checker_fn checker,
             void* ctx, orc_eizo_iter_t* iters, int32_t* num_iters, int nthreads) {
  const int d = p->num_configuration_variables;
  if (d > 16) return -1;
  set_threads(nthreads);
  int F = *num_faces;
  int nit = 0;
  std::vector<float> samples, proj, lo, hi, mid, cols;
  std::vector<float> dist;
  std::vector<uint8_t> flags;
  auto check = [&](const float* q, int64_t n, uint8_t* out) {
    if (checker) return checker(q, n, out, ctx);
    return orc_check_points(p, q, n, ORC_RULE_GPU, voxels, nv, vr, rids, nr, out, nthreads);
  };
  for (uint32_t it = 0; it < o->max_iterations; ++it) {
    float delta_k = (float)(6 * o->delta / (M_PI * M_PI * (it + 1) * (it + 1)));
    uint32_t M = orc_num_samples_unadaptive(o->epsilon, delta_k, o->tau);
    uint32_t N = std::max(M, o->num_particles);
    samples.assign((size_t)N * d, 0.f);
    // chains that fail keep their start point (inside the region)
#pragma omp parallel
    {
      std::vector<float> sl(F), adv(F);
#pragma omp for schedule(static)
      for (int64_t c = 0; c < (int64_t)N; ++c) {
        float x[16];
        const bool ok = run_chain_carried(A, b, F, d, ls, (int)o->mixing_steps, o->seed, (uint32_t)c, 0u, x,
                                          sl.data(), adv.data());
        for (int k = 0; k < d; ++k) samples[(size_t)c * d + k] = ok ? x[k] : ls[k];
      }
    }
    flags.assign(N, 0);
    if (check(samples.data(), N, flags.data())) return -3;
    uint32_t total = 0, first_m = 0;
    cols.clear();
    for (uint32_t s = 0; s < N; ++s) {
      if (!flags[s]) {
        if (total < o->num_particles)
          cols.insert(cols.end(), samples.begin() + (size_t)s * d, samples.begin() + (size_t)(s + 1) * d);
        ++total;
        if (s < M) ++first_m;
      }
    }
    float thr = (1 - o->tau) * o->epsilon * M;
    orc_eizo_iter_t info;
    info.iteration_index = (int32_t)it;
    info.num_samples_drawn = (int32_t)N;
    info.collisions_threshold = (int32_t)thr;
    info.num_collisions_unadaptive = (int32_t)first_m;
    info.num_faces_placed = 0;
    info.num_collisions_updated = 0;
    if ((float)first_m <= thr) {
      if (iters) iters[nit] = info;
      ++nit;
      break;
    }
    uint32_t K = std::min(total, o->num_particles);
    // projection onto the segment, cuda_set_builder_utils.cu:25-67
    proj.assign((size_t)K * d, 0.f);
    dist.assign(K, 0.f);
    float seg2 = 0.f;
    for (int k = 0; k < d; ++k) seg2 = std::fmaf(le[k] - ls[k], le[k] - ls[k], seg2);
    for (uint32_t i = 0; i < K; ++i) {
      const float* c = cols.data() + (size_t)i * d;
      float a = 0.f;
      for (int k = 0; k < d; ++k) a = std::fmaf(c[k] - ls[k], le[k] - ls[k], a);
      float t = std::fmin(std::fmax(a / seg2, 0.0f), 1.0f);
      for (int k = 0; k < d; ++k) proj[(size_t)i * d + k] = std::fmaf(t, le[k], (1.0f - t) * ls[k]);
    }
    // bisection, cuda_edge_inflation_zero_order.cu:215-259
    lo = proj;
    hi.assign(cols.begin(), cols.begin() + (size_t)K * d);
    mid.assign((size_t)K * d, 0.f);
    std::vector<uint8_t> mflags(K);
    for (uint32_t bs = 0; bs < o->bisection_steps; ++bs) {
      for (size_t j = 0; j < (size_t)K * d; ++j) mid[j] = 0.5f * (lo[j] + hi[j]);
      if (check(mid.data(), K, mflags.data())) return -3;
      for (uint32_t i = 0; i < K; ++i) {
        float* dst = mflags[i] ? lo.data() : hi.data();
        std::memcpy(dst + (size_t)i * d, mid.data() + (size_t)i * d, sizeof(float) * d);
        if (!mflags[i]) std::memcpy(cols.data() + (size_t)i * d, mid.data() + (size_t)i * d, sizeof(float) * d);
      }
    }
    // distances to the (pre-bisection) projections, cuda_set_builder_utils.cu:332-345
    for (uint32_t i = 0; i < K; ++i) {
      float s2 = 0.f;
      for (int k = 0; k < d; ++k) {
        float x = cols[(size_t)i * d + k] - proj[(size_t)i * d + k];
        s2 = std::fmaf(x, x, s2);
      }
      dist[i] = std::sqrt(s2);
    }
    // greedy faces, cuda_edge_inflation_zero_order.cu:273-306 and
    // cuda_set_builder_utils.cu:359-424
    uint32_t placed = 0;
    for (; placed < o->max_hyperplanes_per_iteration; ++placed) {
      uint32_t best = 0;
      float bd = FLT_MAX;
      for (uint32_t i = 0; i < K; ++i)
        if (dist[i] < bd) {
          bd = dist[i];
          best = i;
        }
      if (!(bd < FLT_MAX)) break;
      if (F >= capacity) return 2;
      const float* c = cols.data() + (size_t)best * d;
      const float* pr = proj.data() + (size_t)best * d;
      float a[16];
      float n2 = 0.f;
      for (int k = 0; k < d; ++k) {
        a[k] = c[k] - pr[k];
        n2 = std::fmaf(a[k], a[k], n2);
      }
      float nrm = std::sqrt(n2);
      for (int k = 0; k < d; ++k) a[k] = a[k] / nrm;
      float bb = 0.f, v1 = 0.f, v2 = 0.f;
      for (int k = 0; k < d; ++k) {
        bb = std::fmaf(a[k], c[k], bb);
        v1 = std::fmaf(a[k], ls[k], v1);
        v2 = std::fmaf(a[k], le[k], v2);
      }
      bb = bb - o->configuration_margin;
      v1 = v1 - bb;
      v2 = v2 - bb;
      float relax = v2 > v1 ? v2 : v1;
      relax = relax > 0 ? relax : 0;
      bb = bb + relax;
      for (int k = 0; k < d; ++k) A[(int64_t)F * d + k] = a[k];
      b[F] = bb;
      ++F;
      dist[best] = FLT_MAX;
      for (uint32_t i = 0; i < K; ++i) {
        if (dist[i] == FLT_MAX) continue;
        float v = 0.f;
        for (int k = 0; k < d; ++k) v = std::fmaf(a[k], cols[(size_t)i * d + k], v);
        if (v - bb > 0) dist[i] = FLT_MAX;
      }
    }
    info.num_faces_placed = (int32_t)placed;
    info.num_collisions_updated = (int32_t)K;
    if (iters) iters[nit] = info;
    ++nit;
  }
  *num_faces = F;
  if (num_iters) *num_iters = nit;
  return 0;
}

// EditRegionsCuda, cuda_edit_regions.cu:44-301. Collisions are grouped by
// segment in a stable counting order (:85-107); each is projected onto its
// segment (cuda_set_builder_utils.cu:25-67, the projection kernel called at
// :177), bisected towards the projection (:196-225) and measured against it
// (:227-230). Per region the candidates are visited in ascending distance
// (:239-241, std::sort there; equal distances here keep their group order)
// and a face is added for each one that lies strictly inside the region as
// edited so far (:253-259), with the segment relaxation of :262-272.
// Region r's faces are written at row face_offsets[r] + (collisions of the
// segments before r); projections and optimized collisions come out in the
// grouped order. Dot products are accumulated in coordinate order with
// fused multiply-adds. A non-NULL checker replaces the oracle's own point
// check (GPU contact rule). Returns 0, -1 for a dimension above 16, -2 for a
// segment index out of range, -3 if the point check fails.
int orc_edit_regions(const orc_plant_t* p, const float* collisions, const uint32_t* seg, int64_t n,
                     const float* starts, const float* ends, int32_t m, const float* A, const float* b,
                     const int32_t* face_offsets, const float* voxels, int32_t nv, float vr,
                     const int32_t* rids, int32_t nr, float margin, uint32_t steps, float* A_out,
                     float* b_out, int32_t* num_faces, float* proj_out, float* opt_out,
                     orc_checker_fn checker, void* ctx, int nthreads) {
  const int d = p->num_configuration_variables;
  if (d > 16) return -1;
  set_threads(nthreads);
  for (int64_t i = 0; i < n; ++i)
    if (seg[i] >= (uint32_t)m) return -2;
  // stable grouping by segment
  std::vector<int64_t> coff(m + 1, 0);
  for (int64_t i = 0; i < n; ++i) ++coff[seg[i] + 1];
  for (int r = 0; r < m; ++r) coff[r + 1] += coff[r];
  std::vector<int64_t> fill(coff.begin(), coff.end() - 1);
  std::vector<float> cols((size_t)n * d), proj((size_t)n * d), lo, hi, mid((size_t)n * d);
  std::vector<uint32_t> gseg(n);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t j = fill[seg[i]]++;
    std::memcpy(&cols[(size_t)j * d], collisions + (size_t)i * d, sizeof(float) * d);
    gseg[j] = seg[i];
  }
  for (int64_t i = 0; i < n; ++i) {
    const float* ls = starts + (size_t)gseg[i] * d;
    const float* le = ends + (size_t)gseg[i] * d;
    const float* c = &cols[(size_t)i * d];
    float seg2 = 0.f, a = 0.f;
    for (int k = 0; k < d; ++k) {
      seg2 = std::fmaf(le[k] - ls[k], le[k] - ls[k], seg2);
      a = std::fmaf(c[k] - ls[k], le[k] - ls[k], a);
    }
    float t = std::fmin(std::fmax(a / seg2, 0.0f), 1.0f);
    for (int k = 0; k < d; ++k) proj[(size_t)i * d + k] = std::fmaf(t, le[k], (1.0f - t) * ls[k]);
  }
  lo = proj;
  hi = cols;
  std::vector<uint8_t> flags(n);
  for (uint32_t s = 0; s < steps; ++s) {
    for (size_t j = 0; j < (size_t)n * d; ++j) mid[j] = 0.5f * (lo[j] + hi[j]);
    const int rc = checker ? checker(mid.data(), n, flags.data(), ctx)
                           : orc_check_points(p, mid.data(), n, ORC_RULE_GPU, voxels, nv, vr, rids, nr,
                                              flags.data(), nthreads);
    if (rc) return -3;
    for (int64_t i = 0; i < n; ++i) {
      float* dst = flags[i] ? lo.data() : hi.data();
      std::memcpy(dst + (size_t)i * d, &mid[(size_t)i * d], sizeof(float) * d);
      if (!flags[i]) std::memcpy(&cols[(size_t)i * d], &mid[(size_t)i * d], sizeof(float) * d);
    }
  }
  std::vector<float> dist(n);
  for (int64_t i = 0; i < n; ++i) {
    float s2 = 0.f;
    for (int k = 0; k < d; ++k) {
      float x = cols[(size_t)i * d + k] - proj[(size_t)i * d + k];
      s2 = std::fmaf(x, x, s2);
    }
    dist[i] = std::sqrt(s2);
  }
  std::memcpy(proj_out, proj.data(), sizeof(float) * n * d);
  std::memcpy(opt_out, cols.data(), sizeof(float) * n * d);
  for (int r = 0; r < m; ++r) {
    const int64_t F0 = face_offsets[r + 1] - face_offsets[r];
    const int64_t row0 = face_offsets[r] + coff[r];
    float* Ao = A_out + (size_t)row0 * d;
    float* bo = b_out + row0;
    std::memcpy(Ao, A + (size_t)face_offsets[r] * d, sizeof(float) * F0 * d);
    std::memcpy(bo, b + face_offsets[r], sizeof(float) * F0);
    int64_t F = F0;
    std::vector<int64_t> order;
    for (int64_t i = coff[r]; i < coff[r + 1]; ++i)
      if (dist[i] < FLT_MAX) order.push_back(i);
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return dist[x] < dist[y]; });
    const float* ls = starts + (size_t)r * d;
    const float* le = ends + (size_t)r * d;
    for (int64_t i : order) {
      const float* c = &cols[(size_t)i * d];
      bool inside = true;
      for (int64_t f = 0; f < F && inside; ++f) {
        float v = 0.f;
        for (int k = 0; k < d; ++k) v = std::fmaf(Ao[(size_t)f * d + k], c[k], v);
        if (!(v - bo[f] < 0.f)) inside = false;
      }
      if (!inside) continue;
      const float* pr = &proj[(size_t)i * d];
      float a[16];
      float n2 = 0.f;
      for (int k = 0; k < d; ++k) {
        a[k] = c[k] - pr[k];
        n2 = std::fmaf(a[k], a[k], n2);
      }
      if (n2 > 0.f) {
        float nrm = std::sqrt(n2);
        for (int k = 0; k < d; ++k) a[k] = a[k] / nrm;
      }
      float bb = 0.f, v1 = 0.f, v2 = 0.f;
      for (int k = 0; k < d; ++k) {
        bb = std::fmaf(a[k], c[k], bb);
        v1 = std::fmaf(a[k], ls[k], v1);
        v2 = std::fmaf(a[k], le[k], v2);
      }
      bb = bb - margin;
      v1 = v1 - bb;
      v2 = v2 - bb;
      float relax = std::max(v1, v2);
      if (relax > 0) bb = (float)((double)bb + ((double)relax + 2e-6));
      for (int k = 0; k < d; ++k) Ao[(size_t)F * d + k] = a[k];
      bo[F] = bb;
      ++F;
    }
    num_faces[r] = (int32_t)F;
  }
  return 0;
}

}  // extern "C"
