// plant.cu -- host preprocessing of a MinimalPlant into the device layout of
// csd_device.cuh, and the plant handle's lifetime.
//
// Reference: the MinimalPlant is copied whole to the GPU on every call
// (csdecomp/src/plant/cuda_collision_checker.cu:458-462) and FK walks every
// joint, fixed ones included (cuda_forward_kinematics.cu:14-57). Here the
// tree is flattened once: fixed-joint chains are pre-composed in FP64,
// world-fixed geometry is posed once, and the pair list is split into
// moving-sphere x static tiles (lane masks) and a generic remainder.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>

#include "csd_internal.h"

namespace csd {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

csd_status_t DevBuf::reserve(size_t n) {
  if (n <= bytes && ptr) return CSD_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
  size_t nb = std::max<size_t>(n, 256);
  CSD_CUDA_TRY(cudaMalloc(&ptr, nb));
  bytes = nb;
  return CSD_OK;
}

DevBuf::~DevBuf() {
  if (ptr) cudaFree(ptr);
}

int device_sm_count() {
  static std::mutex mu;
  static int cache[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (dev < 0 || dev >= 64) return 148;
  if (!cache[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = n > 0 ? n : 148;
  }
  return cache[dev];
}

namespace {

// Bits 0..9 of v spread to bits 0, 3, 6, ..., 27 (one coordinate of a 30-bit
// Morton code).
uint32_t spread10(uint32_t v) {
  v &= 1023u;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

struct X4 {  // rigid transform in FP64: R column-major, t
  double R[9];
  double t[3];
};

X4 ident() {
  X4 x{};
  x.R[0] = x.R[4] = x.R[8] = 1.0;
  return x;
}

X4 from_colmajor(const float* m) {
  X4 x;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) x.R[c * 3 + r] = m[c * 4 + r];
  for (int r = 0; r < 3; ++r) x.t[r] = m[12 + r];
  return x;
}

X4 mul(const X4& a, const X4& b) {
  X4 o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += a.R[k * 3 + r] * b.R[c * 3 + k];
      o.R[c * 3 + r] = s;
    }
  for (int r = 0; r < 3; ++r) {
    double s = a.t[r];
    for (int k = 0; k < 3; ++k) s += a.R[k * 3 + r] * b.t[k];
    o.t[r] = s;
  }
  return o;
}

// World-format (16 floats) pose of a geometry from its FP64 world transform.
void world_pose(int type, const float* dims, const X4& X, float* out) {
  for (int i = 0; i < 16; ++i) out[i] = 0.f;
  if (type == G_SPHERE) {
    for (int r = 0; r < 3; ++r) out[r] = (float)X.t[r];
    out[3] = dims[0];
  } else if (type == G_CAPSULE) {
    for (int r = 0; r < 3; ++r) {
      out[r] = (float)X.t[r];
      out[4 + r] = (float)X.R[6 + r];
    }
    out[3] = dims[0];
    out[7] = 0.5f * dims[1];
  } else {
    for (int a = 0; a < 3; ++a) {
      double q = 0;
      for (int r = 0; r < 3; ++r) {
        out[4 * a + r] = (float)X.R[a * 3 + r];
        q += X.R[a * 3 + r] * X.t[r];
      }
      out[4 * a + 3] = (float)(-q);
      out[12 + a] = 0.5f * dims[a];
    }
  }
}

// FP64 collision test of two world-fixed geometries (evaluated once).
struct DGeom {
  int type;
  double c[3], ax[3][3], h[3], r, hl;
};

DGeom dgeom(int type, const float* dims, const X4& X) {
  DGeom g{};
  g.type = type;
  for (int r = 0; r < 3; ++r) g.c[r] = X.t[r];
  for (int a = 0; a < 3; ++a)
    for (int r = 0; r < 3; ++r) g.ax[a][r] = X.R[a * 3 + r];
  g.r = dims[0];
  g.hl = 0.5 * dims[1];
  for (int a = 0; a < 3; ++a) g.h[a] = 0.5 * dims[a];
  return g;
}

double dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

double point_box_d2(const double* p, const DGeom& B) {
  double d[3] = {p[0] - B.c[0], p[1] - B.c[1], p[2] - B.c[2]};
  double s = 0;
  for (int a = 0; a < 3; ++a) {
    double e = std::max(std::fabs(dot(B.ax[a], d)) - B.h[a], 0.0);
    s += e * e;
  }
  return s;
}

double point_seg_d2(const double* p, const DGeom& C) {
  double d[3] = {p[0] - C.c[0], p[1] - C.c[1], p[2] - C.c[2]};
  double t = std::max(-C.hl, std::min(dot(d, C.ax[2]), C.hl));
  double e[3] = {d[0] - t * C.ax[2][0], d[1] - t * C.ax[2][1], d[2] - t * C.ax[2][2]};
  return dot(e, e);
}

// distance^2 from a capsule segment to a geometry by dense sampling refined
// with a golden-section search (convex in t); exact enough for a one-off test.
double seg_to_d2(const DGeom& C, const DGeom& O) {
  auto f = [&](double t) {
    double p[3] = {C.c[0] + t * C.ax[2][0], C.c[1] + t * C.ax[2][1], C.c[2] + t * C.ax[2][2]};
    if (O.type == G_SPHERE) {
      double d[3] = {p[0] - O.c[0], p[1] - O.c[1], p[2] - O.c[2]};
      return dot(d, d);
    }
    if (O.type == G_BOX) return point_box_d2(p, O);
    return point_seg_d2(p, O);
  };
  double lo = -C.hl, hi = C.hl;
  for (int it = 0; it < 200; ++it) {
    double m1 = lo + (hi - lo) / 3, m2 = hi - (hi - lo) / 3;
    if (f(m1) < f(m2))
      hi = m2;
    else
      lo = m1;
  }
  return f(0.5 * (lo + hi));
}

bool static_pair_hit(const DGeom& A, const DGeom& B) {
  if (A.type == G_SPHERE && B.type == G_SPHERE) {
    double d[3] = {A.c[0] - B.c[0], A.c[1] - B.c[1], A.c[2] - B.c[2]};
    return dot(d, d) < (A.r + B.r) * (A.r + B.r);
  }
  if (A.type == G_SPHERE && B.type == G_BOX) return point_box_d2(A.c, B) < A.r * A.r;
  if (A.type == G_BOX && B.type == G_SPHERE) return point_box_d2(B.c, A) < B.r * B.r;
  if (A.type == G_CAPSULE) {
    double rr = A.r + (B.type == G_BOX ? 0.0 : B.r);
    return seg_to_d2(A, B) < rr * rr;
  }
  if (B.type == G_CAPSULE) return static_pair_hit(B, A);
  // box-box SAT
  double axes[15][3];
  int n = 0;
  for (int a = 0; a < 3; ++a) {
    for (int r = 0; r < 3; ++r) axes[n][r] = A.ax[a][r];
    ++n;
    for (int r = 0; r < 3; ++r) axes[n][r] = B.ax[a][r];
    ++n;
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double* a = A.ax[i];
      const double* b = B.ax[j];
      axes[n][0] = a[1] * b[2] - a[2] * b[1];
      axes[n][1] = a[2] * b[0] - a[0] * b[2];
      axes[n][2] = a[0] * b[1] - a[1] * b[0];
      ++n;
    }
  double d[3] = {A.c[0] - B.c[0], A.c[1] - B.c[1], A.c[2] - B.c[2]};
  for (int s = 0; s < 15; ++s) {
    double lhs = std::fabs(dot(d, axes[s]));
    double rhs = 0;
    for (int a = 0; a < 3; ++a) rhs += A.h[a] * std::fabs(dot(A.ax[a], axes[s])) + B.h[a] * std::fabs(dot(B.ax[a], axes[s]));
    if (lhs > rhs) return false;
  }
  return true;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace csd

csd_plant_s::~csd_plant_s() {
  if (blob) cudaFree(blob);
}

using namespace csd;

extern "C" {

const char* csd_last_error(void) { return csd::g_err.c_str(); }

int32_t csd_version(void) { return 10000; }

csd_status_t csd_plant_create(const csd_plant_desc_t* d, csd_plant_t* out) {
  CSD_CHECK(d && out, CSD_ERR_INVALID, "null argument");
  *out = nullptr;
  const int J = d->num_joints, L = d->num_links, D = d->num_configuration_variables, G = d->num_geometries,
            P = d->num_collision_pairs;
  CSD_CHECK(J >= 0 && L >= 1 && D >= 0 && G >= 0 && P >= 0, CSD_ERR_INVALID, "negative plant sizes");
  CSD_CHECK(D <= kMaxDim, CSD_ERR_CAPACITY, "more than 16 configuration variables");
  CSD_CHECK(J == 0 || (d->joint_type && d->joint_parent_link && d->joint_child_link && d->joint_idx_to_config_idx &&
                       d->joint_traversal_sequence && d->joint_X_PL_J && d->joint_axis),
            CSD_ERR_INVALID, "null joint table");
  CSD_CHECK(G == 0 || (d->geom_type && d->geom_link_index && d->geom_dimensions && d->geom_X_L_B), CSD_ERR_INVALID,
            "null geometry table");
  CSD_CHECK(P == 0 || d->collision_pairs_flat, CSD_ERR_INVALID, "null pair table");
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    set_error("no CUDA device");
    return CSD_ERR_NO_DEVICE;
  }

  // ---- tree flattening
  std::vector<int> slot(L, -2);
  std::vector<X4> X(L, ident());
  slot[0] = -1;
  std::vector<FkJoint> fk;
  std::vector<char> seen(J, 0);
  for (int t = 0; t < J; ++t) {
    int j = d->joint_traversal_sequence[t];
    CSD_CHECK(j >= 0 && j < J && !seen[j], CSD_ERR_INVALID, "bad joint traversal sequence");
    seen[j] = 1;
    int pl = d->joint_parent_link[j], cl = d->joint_child_link[j], ty = d->joint_type[j];
    CSD_CHECK(pl >= 0 && pl < L && cl >= 0 && cl < L, CSD_ERR_INVALID, "joint link index out of range");
    CSD_CHECK(ty >= J_FIXED && ty <= J_PRISMATIC, CSD_ERR_INVALID, "bad joint type");
    CSD_CHECK(slot[pl] != -2, CSD_ERR_INVALID, "traversal visits a child before its parent");
    X4 xp = mul(X[pl], from_colmajor(d->joint_X_PL_J + 16 * j));
    if (ty == J_FIXED) {
      slot[cl] = slot[pl];
      X[cl] = xp;
      continue;
    }
    int qi = d->joint_idx_to_config_idx[j];
    CSD_CHECK(qi >= 0 && qi < D, CSD_ERR_INVALID, "joint configuration index out of range");
    CSD_CHECK((int)fk.size() < kMaxSlots, CSD_ERR_CAPACITY, "more than 32 moving joints");
    FkJoint f{};
    f.type = ty;
    f.parent = slot[pl];
    f.child = (int)fk.size();
    f.qidx = qi;
    double a[3] = {d->joint_axis[3 * j], d->joint_axis[3 * j + 1], d->joint_axis[3 * j + 2]};
    double Ra[3];
    for (int r = 0; r < 3; ++r) Ra[r] = xp.R[r] * a[0] + xp.R[3 + r] * a[1] + xp.R[6 + r] * a[2];
    if (ty == J_REVOLUTE) {
      // R(q) = Rp (c I + s [a]x + (1-c) a a^T) = c (Rp - Ra a^T) + s Rp [a]x + Ra a^T
      double K[9] = {0, a[2], -a[1], -a[2], 0, a[0], a[1], -a[0], 0};  // [a]x column-major
      for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) {
          double T = Ra[r] * a[c];
          double S = 0;
          for (int k = 0; k < 3; ++k) S += xp.R[k * 3 + r] * K[c * 3 + k];
          f.P[c * 3 + r] = (float)(xp.R[c * 3 + r] - T);
          f.S[c * 3 + r] = (float)S;
          f.T[c * 3 + r] = (float)T;
        }
    } else {
      for (int i = 0; i < 9; ++i) f.P[i] = (float)xp.R[i];
      for (int r = 0; r < 3; ++r) f.v[r] = (float)Ra[r];
    }
    for (int r = 0; r < 3; ++r) f.t[r] = (float)xp.t[r];
    fk.push_back(f);
    slot[cl] = f.child;
    X[cl] = ident();
  }

  // ---- geometries
  std::unique_ptr<csd_plant_s> h(new csd_plant_s());
  cudaGetDevice(&h->device);
  HostPlant& hp = h->host;
  hp.dim = D;
  hp.num_links = L;
  hp.moving_of_geom.assign(G, -1);
  hp.static_of_geom.assign(G, -1);
  hp.geom_type.resize(G);
  std::vector<X4> gX(G);
  std::vector<int> mov_sph, mov_cap, mov_box, st_sph, st_box, st_cap;
  for (int g = 0; g < G; ++g) {
    int ty = d->geom_type[g], l = d->geom_link_index[g];
    if (ty == G_CYLINDER) {
      set_error("Cylinders are not supported (collision_checker.cpp:104-107).");
      return CSD_ERR_UNSUPPORTED;
    }
    CSD_CHECK(ty == G_BOX || ty == G_SPHERE || ty == G_CAPSULE, CSD_ERR_INVALID, "bad geometry type");
    CSD_CHECK(l >= 0 && l < L && slot[l] != -2, CSD_ERR_INVALID, "geometry on an unknown or unreachable link");
    hp.geom_type[g] = ty;
    gX[g] = mul(X[l], from_colmajor(d->geom_X_L_B + 16 * g));
    bool moving = slot[l] >= 0;
    auto& lst = moving ? (ty == G_SPHERE ? mov_sph : ty == G_CAPSULE ? mov_cap : mov_box)
                       : (ty == G_SPHERE ? st_sph : ty == G_BOX ? st_box : st_cap);
    lst.push_back(g);
  }
  std::vector<int> mov_order(mov_sph);
  mov_order.insert(mov_order.end(), mov_cap.begin(), mov_cap.end());
  mov_order.insert(mov_order.end(), mov_box.begin(), mov_box.end());
  // Statics of each class in the Morton order of their world positions, so
  // that the broad phase's groups of 32 consecutive statics are spatially
  // compact and a group sphere far from every link culls the whole group.
  // (Which static comes first changes no verdict: a configuration collides
  // if any pair does.)
  {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (const std::vector<int>* lst : {&st_sph, &st_box, &st_cap})
      for (int g : *lst)
        for (int a = 0; a < 3; ++a) {
          lo[a] = std::min(lo[a], gX[g].t[a]);
          hi[a] = std::max(hi[a], gX[g].t[a]);
        }
    auto code = [&](int g) {
      uint32_t c = 0;
      for (int a = 0; a < 3; ++a) {
        const double u = hi[a] > lo[a] ? (gX[g].t[a] - lo[a]) / (hi[a] - lo[a]) : 0.0;
        c |= spread10((uint32_t)std::min(1023.0, std::max(0.0, u * 1023.0))) << a;
      }
      return c;
    };
    for (std::vector<int>* lst : {&st_sph, &st_box, &st_cap})
      std::stable_sort(lst->begin(), lst->end(), [&](int x, int y) { return code(x) < code(y); });
  }
  // world boxes whose axes are exactly the world axes get the aligned fast path
  std::vector<int> st_abox, st_rbox;
  for (int g : st_box) {
    bool aligned = true;
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r)
        if ((float)gX[g].R[c * 3 + r] != (c == r ? 1.f : 0.f)) aligned = false;
    (aligned ? st_abox : st_rbox).push_back(g);
  }
  std::vector<int> st_order(st_sph);
  st_order.insert(st_order.end(), st_abox.begin(), st_abox.end());
  st_order.insert(st_order.end(), st_rbox.begin(), st_rbox.end());
  st_order.insert(st_order.end(), st_cap.begin(), st_cap.end());
  int pose_words = 0;
  for (size_t m = 0; m < mov_order.size(); ++m) {
    int g = mov_order[m];
    const float* dm = d->geom_dimensions + 3 * g;
    MovingGeom mg{};
    mg.type = d->geom_type[g];
    mg.slot = slot[d->geom_link_index[g]];
    mg.pose_off = pose_words;
    pose_words += mg.type == G_SPHERE ? 4 : mg.type == G_CAPSULE ? 8 : 16;
    mg.r = dm[0];
    mg.hl = 0.5f * dm[1];
    for (int r = 0; r < 3; ++r) {
      mg.p[r] = (float)gX[g].t[r];
      mg.z[r] = (float)gX[g].R[6 + r];
      mg.h[r] = 0.5f * dm[r];
    }
    for (int i = 0; i < 9; ++i) mg.R[i] = (float)gX[g].R[i];
    hp.moving.push_back(mg);
    hp.moving_of_geom[g] = (int)m;
  }
  hp.statics.assign(st_order.size() * 16, 0.f);
  for (size_t s = 0; s < st_order.size(); ++s) {
    int g = st_order[s];
    world_pose(d->geom_type[g], d->geom_dimensions + 3 * g, gX[g], hp.statics.data() + 16 * s);
    hp.static_type.push_back(d->geom_type[g]);
    hp.static_of_geom[g] = (int)s;
  }

  // ---- pairs
  const int S = (int)st_order.size();
  const int nmsph = (int)mov_sph.size();
  const int T = (nmsph + kWarp - 1) / kWarp;
  const int cls_begin[5] = {0, (int)st_sph.size(), (int)(st_sph.size() + st_abox.size()),
                            (int)(st_sph.size() + st_abox.size() + st_rbox.size()), S};
  std::vector<uint32_t> masks((size_t)T * S, 0u);               // tile x static
  std::vector<uint32_t> self_masks((size_t)T * nmsph, 0u);      // tile x moving-sphere partner
  std::vector<GenericPair> generic;
  std::vector<GenericPair> self_pairs;  // moving sphere x moving sphere
  int always = 0, tile_pairs = 0;
  auto ref = [&](int g) -> uint32_t {
    int m = hp.moving_of_geom[g];
    return m >= 0 ? (uint32_t)m : (0x80000000u | (uint32_t)hp.static_of_geom[g]);
  };
  for (int k = 0; k < P; ++k) {
    int a = d->collision_pairs_flat[2 * k], b = d->collision_pairs_flat[2 * k + 1];
    CSD_CHECK(a >= 0 && a < G && b >= 0 && b < G, CSD_ERR_INVALID, "collision pair index out of range");
    int ma = hp.moving_of_geom[a], mb = hp.moving_of_geom[b];
    if (ma < 0 && mb < 0) {
      const float* da = d->geom_dimensions + 3 * a;
      const float* db = d->geom_dimensions + 3 * b;
      if (static_pair_hit(dgeom(d->geom_type[a], da, gX[a]), dgeom(d->geom_type[b], db, gX[b]))) always = 1;
      continue;
    }
    if ((ma >= 0 && mb < 0 && ma < nmsph) || (mb >= 0 && ma < 0 && mb < nmsph)) {
      int m = ma >= 0 ? ma : mb;
      int st = ma >= 0 ? hp.static_of_geom[b] : hp.static_of_geom[a];
      uint32_t& w = masks[(size_t)(m / kWarp) * S + st];
      if (!(w & (1u << (m % kWarp)))) ++tile_pairs;
      w |= 1u << (m % kWarp);
      continue;
    }
    if (ma >= 0 && mb >= 0 && ma < nmsph && mb < nmsph && ma != mb) {
      int lo = std::min(ma, mb), hi = std::max(ma, mb);
      self_masks[(size_t)(lo / kWarp) * nmsph + hi] |= 1u << (lo % kWarp);
      self_pairs.push_back({(uint32_t)lo, (uint32_t)hi});
      continue;
    }
    // generic: the moving geometry first
    if (ma < 0 || (mb >= 0 && mb < ma)) std::swap(a, b);
    generic.push_back({ref(a), ref(b)});
  }
  // Self pairs as masked tile entries cost about one warp pass per (tile,
  // partner) with a nonzero mask; as generic pairs, one pass per 32 pairs
  // with two pose loads each. Keep the cheaper form.
  {
    size_t entries_needed = 0;
    for (uint32_t w : self_masks) entries_needed += w != 0u;
    const size_t generic_passes = (self_pairs.size() + kWarp - 1) / kWarp;
    if (15 * entries_needed > 18 * generic_passes) {
      std::fill(self_masks.begin(), self_masks.end(), 0u);
      generic.insert(generic.end(), self_pairs.begin(), self_pairs.end());
    }
  }
  auto type_of_ref = [&](uint32_t r) {
    return (r & 0x80000000u) ? hp.static_type[r & 0x7fffffffu] : hp.moving[r].type;
  };
  auto seg_key = [&](const GenericPair& x) {
    return ((x.b >> 31) * 16 + type_of_ref(x.a) * 4 + type_of_ref(x.b));
  };
  // by segment, then by the moving geometry's slot and the partner (so that
  // consecutive pairs mostly share a link pair for the broad phase)
  auto slot_of_ref = [&](uint32_t r) { return (r & 0x80000000u) ? -1 : hp.moving[r].slot; };
  std::stable_sort(generic.begin(), generic.end(), [&](const GenericPair& x, const GenericPair& y) {
    const uint32_t kx = seg_key(x), ky = seg_key(y);
    if (kx != ky) return kx < ky;
    const int ax = slot_of_ref(x.a), ay = slot_of_ref(y.a);
    if (ax != ay) return ax < ay;
    return slot_of_ref(x.b) < slot_of_ref(y.b);
  });
  std::vector<GenSeg> segs;
  std::vector<PairRun> runs;  // moving-moving segments split where the (slot a, slot b) pair changes
  for (size_t i = 0; i < generic.size();) {
    size_t j = i;
    while (j < generic.size() && seg_key(generic[j]) == seg_key(generic[i])) ++j;
    GenSeg sg{};
    sg.begin = (int)i;
    sg.end = (int)j;
    sg.ta = type_of_ref(generic[i].a);
    sg.tb = type_of_ref(generic[i].b);
    sg.b_static = (int)(generic[i].b >> 31);
    sg.run_begin = (int)runs.size();
    if (!sg.b_static)
      for (size_t r = i; r < j;) {
        size_t e = r;
        const int sa = slot_of_ref(generic[r].a), sb = slot_of_ref(generic[r].b);
        while (e < j && slot_of_ref(generic[e].a) == sa && slot_of_ref(generic[e].b) == sb) ++e;
        runs.push_back({(int)r, (int)e, sa, sb});
        r = e;
      }
    sg.run_end = (int)runs.size();
    segs.push_back(sg);
    i = j;
  }
  std::vector<TileInfo> tiles(T);
  std::vector<TileEntry> entries;
  for (int t = 0; t < T; ++t) {
    int lanes = std::min(kWarp, nmsph - t * kWarp);
    uint32_t valid = lanes == 32 ? 0xffffffffu : ((1u << lanes) - 1u);
    TileInfo ti{};
    for (int c = 0; c < 4; ++c) {
      bool dense = true;
      for (int st = cls_begin[c]; st < cls_begin[c + 1]; ++st)
        if (masks[(size_t)t * S + st] != valid) dense = false;
      ti.dense[c] = dense ? 1 : 0;
      ti.ent[c] = (int)entries.size();
      if (!dense)
        for (int st = cls_begin[c]; st < cls_begin[c + 1]; ++st)
          if (masks[(size_t)t * S + st]) entries.push_back({(uint32_t)st, masks[(size_t)t * S + st]});
    }
    ti.ent[4] = (int)entries.size();
    ti.self_begin = (int)entries.size();
    for (int m2 = 0; m2 < nmsph; ++m2)
      if (self_masks[(size_t)t * nmsph + m2]) entries.push_back({(uint32_t)m2, self_masks[(size_t)t * nmsph + m2]});
    ti.self_end = (int)entries.size();
    tiles[t] = ti;
  }
  hp.num_tile_pairs = tile_pairs;
  for (const FkJoint& f : fk)
    hp.flops_fk += f.type == J_REVOLUTE ? (f.parent < 0 ? kFlopFkRootRevolute : kFlopFkRevolute)
                                        : (f.parent < 0 ? kFlopFkRootPrismatic : kFlopFkPrismatic);
  for (const MovingGeom& g : hp.moving)
    hp.flops_place += g.type == G_SPHERE ? kFlopPlaceSphere : g.type == G_CAPSULE ? kFlopPlaceCapsule : kFlopPlaceBox;
  for (int t = 0; t < T; ++t) {
    int lanes = std::min(kWarp, nmsph - t * kWarp);
    for (int c = 0; c < 4; ++c)
      for (int st = cls_begin[c]; st < cls_begin[c + 1]; ++st) {
        uint32_t w = masks[(size_t)t * S + st];
        int cnt = tiles[t].dense[c] ? lanes : __builtin_popcount(w);
        hp.flops_pairs += cnt * (c == SC_ABOX ? kFlopSphABox : pair_flops(G_SPHERE, hp.static_type[st]));
      }
    for (int e = tiles[t].self_begin; e < tiles[t].self_end; ++e)
      hp.flops_pairs += __builtin_popcount(entries[e].mask) * kFlopSphSph;
  }
  for (const GenericPair& gp : generic) hp.flops_pairs += pair_flops(type_of_ref(gp.a), type_of_ref(gp.b));
  // axis-aligned box table [p 0 | h 0]
  std::vector<float> aabb(st_abox.size() * 8, 0.f);
  for (size_t i = 0; i < st_abox.size(); ++i) {
    const float* W = hp.statics.data() + 16 * (cls_begin[SC_ABOX] + i);
    for (int a = 0; a < 3; ++a) {
      aabb[8 * i + a] = -W[4 * a + 3];
      aabb[8 * i + 4 + a] = W[12 + a];
    }
  }

  // ---- broad-phase tables. Bounding spheres (FP64, then padded by a relative
  // 1e-6 and 1e-4 m so that FP32 evaluation never culls a pair closer than
  // that): per slot over its geometries in the slot frame, per static in the
  // world.
  const int NSL = (int)fk.size();
  std::vector<float> slot_bs((size_t)NSL * 4, 0.f);
  {
    std::vector<std::vector<std::array<double, 4>>> pts(std::max(NSL, 1));
    for (const MovingGeom& g : hp.moving) {
      auto add = [&](double x, double y, double z, double r) { pts[g.slot].push_back({x, y, z, r}); };
      if (g.type == G_SPHERE) {
        add(g.p[0], g.p[1], g.p[2], g.r);
      } else if (g.type == G_CAPSULE) {
        for (int sg = -1; sg <= 1; sg += 2)
          add(g.p[0] + sg * g.hl * g.z[0], g.p[1] + sg * g.hl * g.z[1], g.p[2] + sg * g.hl * g.z[2], g.r);
      } else {
        for (int c = 0; c < 8; ++c) {
          double v[3] = {g.p[0], g.p[1], g.p[2]};
          for (int a = 0; a < 3; ++a) {
            const double e = ((c >> a) & 1 ? 1.0 : -1.0) * g.h[a];
            for (int r = 0; r < 3; ++r) v[r] += g.R[3 * a + r] * e;
          }
          add(v[0], v[1], v[2], 0.0);
        }
      }
    }
    for (int k = 0; k < NSL; ++k) {
      if (pts[k].empty()) {
        slot_bs[4 * k + 3] = -1.f;
        continue;
      }
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (auto& q : pts[k])
        for (int a = 0; a < 3; ++a) {
          lo[a] = std::min(lo[a], q[a] - q[3]);
          hi[a] = std::max(hi[a], q[a] + q[3]);
        }
      double c[3], rad = 0;
      for (int a = 0; a < 3; ++a) c[a] = 0.5 * (lo[a] + hi[a]);
      for (auto& q : pts[k])
        rad = std::max(rad, std::sqrt((q[0] - c[0]) * (q[0] - c[0]) + (q[1] - c[1]) * (q[1] - c[1]) +
                                      (q[2] - c[2]) * (q[2] - c[2])) + q[3]);
      for (int a = 0; a < 3; ++a) slot_bs[4 * k + a] = (float)c[a];
      slot_bs[4 * k + 3] = (float)(rad * (1 + 1e-6) + 1e-4);
    }
  }
  std::vector<float> static_bs((size_t)S * 4, 0.f);
  for (int st = 0; st < S; ++st) {
    const float* W = hp.statics.data() + 16 * st;
    double c[3] = {W[0], W[1], W[2]}, rad;
    const int ty = hp.static_type[st];
    if (ty == G_SPHERE) {
      rad = W[3];
    } else if (ty == G_CAPSULE) {
      rad = (double)W[3] + W[7];
    } else {  // box rows [axis_i | -axis_i . centre]: centre = sum_i (axis_i . centre) axis_i
      for (int r = 0; r < 3; ++r) c[r] = 0;
      for (int a = 0; a < 3; ++a)
        for (int r = 0; r < 3; ++r) c[r] += -(double)W[4 * a + 3] * W[4 * a + r];
      rad = std::sqrt((double)W[12] * W[12] + (double)W[13] * W[13] + (double)W[14] * W[14]);
    }
    for (int a = 0; a < 3; ++a) static_bs[4 * st + a] = (float)c[a];
    static_bs[4 * st + 3] = (float)(rad * (1 + 1e-6) + 1e-4);
  }
  // group spheres: one per 32 consecutive statics, enclosing their bounding
  // spheres (FP64, padded again by a relative 1e-6 and 1e-4 m)
  const int NG = (S + kWarp - 1) / kWarp;
  std::vector<float> group_bs((size_t)std::max(NG, 0) * 4, 0.f);
  for (int g = 0; g < NG; ++g) {
    const int s0 = g * kWarp, s1 = std::min(S, s0 + kWarp);
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, c[3], rad = 0;
    for (int st = s0; st < s1; ++st)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], (double)static_bs[4 * st + a] - static_bs[4 * st + 3]);
        hi[a] = std::max(hi[a], (double)static_bs[4 * st + a] + static_bs[4 * st + 3]);
      }
    for (int a = 0; a < 3; ++a) c[a] = 0.5 * (lo[a] + hi[a]);
    for (int st = s0; st < s1; ++st) {
      const double dx = static_bs[4 * st] - c[0], dy = static_bs[4 * st + 1] - c[1], dz = static_bs[4 * st + 2] - c[2];
      rad = std::max(rad, std::sqrt(dx * dx + dy * dy + dz * dz) + static_bs[4 * st + 3]);
    }
    for (int a = 0; a < 3; ++a) group_bs[4 * g + a] = (float)c[a];
    group_bs[4 * g + 3] = (float)(rad * (1 + 1e-6) + 1e-4);
  }
  // Reach masks: for any configuration, slot k's bounding sphere stays within
  // reach[k] of a world-fixed point root[k] (its chain's first joint origin; a
  // child frame's origin lies |t| from its parent's, whatever the revolute
  // angles; a prismatic joint's travel is unbounded, so its subtree gets no
  // bound). A static whose sphere is farther from root[k] than reach[k] plus its
  // radius can never be near slot k; group g's mask holds the slots that can
  // reach some member, and the broad phase tests the others against no static
  // of the group (padded as the spheres; verdicts unchanged).
  std::vector<uint32_t> group_mask((size_t)std::max(NG, 0), 0u);
  {
    std::vector<double> reach(NSL, 0.0), root((size_t)NSL * 3, 0.0);
    std::vector<char> bounded(NSL, 1);
    for (int k = 0; k < NSL; ++k) {
      const FkJoint& f = fk[k];
      const double tl = std::sqrt((double)f.t[0] * f.t[0] + (double)f.t[1] * f.t[1] + (double)f.t[2] * f.t[2]);
      if (f.parent < 0) {
        for (int a = 0; a < 3; ++a) root[3 * k + a] = f.t[a];
        reach[k] = 0.0;
        bounded[k] = f.type != J_PRISMATIC;
      } else {
        for (int a = 0; a < 3; ++a) root[3 * k + a] = root[3 * f.parent + a];
        reach[k] = reach[f.parent] + tl;
        bounded[k] = bounded[f.parent] && f.type != J_PRISMATIC;
      }
    }
    for (int g = 0; g < NG; ++g)
      for (int st = g * kWarp; st < std::min(S, g * kWarp + kWarp); ++st)
        for (int k = 0; k < NSL; ++k) {
          if (slot_bs[4 * k + 3] < 0.f) continue;  // no geometry on the slot
          if (!bounded[k]) {
            group_mask[g] |= 1u << k;
            continue;
          }
          const double ck = std::sqrt((double)slot_bs[4 * k] * slot_bs[4 * k] +
                                      (double)slot_bs[4 * k + 1] * slot_bs[4 * k + 1] +
                                      (double)slot_bs[4 * k + 2] * slot_bs[4 * k + 2]);
          double d2 = 0.0;
          for (int a = 0; a < 3; ++a) {
            const double x = (double)static_bs[4 * st + a] - root[3 * k + a];
            d2 += x * x;
          }
          const double lim = (reach[k] + ck + slot_bs[4 * k + 3] + static_bs[4 * st + 3]) * (1 + 1e-6) + 1e-4;
          if (std::sqrt(d2) <= lim) group_mask[g] |= 1u << k;
        }
  }
  const size_t gm_bytes = ((size_t)std::max(NG, 0) * sizeof(uint32_t) + 15) & ~size_t(15);
  std::vector<uint8_t> moving_slot(std::max<size_t>(hp.moving.size(), 1), 0);
  for (size_t m = 0; m < hp.moving.size(); ++m) moving_slot[m] = (uint8_t)hp.moving[m].slot;

  // ---- FK output tables
  std::vector<int> link_slot(L);
  std::vector<float> link_fixed((size_t)L * 12, 0.f);
  for (int l = 0; l < L; ++l) {
    link_slot[l] = slot[l];
    for (int i = 0; i < 9; ++i) link_fixed[(size_t)l * 12 + i] = (float)X[l].R[i];
    for (int r = 0; r < 3; ++r) link_fixed[(size_t)l * 12 + 9 + r] = (float)X[l].t[r];
  }

  // ---- upload
  size_t off = 0;
  auto section = [&](size_t bytes) {
    size_t o = off;
    off = align256(off + std::max<size_t>(bytes, 16));
    return o;
  };
  size_t o_fk = section(fk.size() * sizeof(FkJoint));
  size_t o_mv = section(hp.moving.size() * sizeof(MovingGeom));
  // staged region: statics | aligned boxes | static spheres | slot spheres | group spheres | group reach
  // masks | geometry slots (16-byte padded)
  const size_t ms_bytes = (moving_slot.size() + 15) & ~size_t(15);
  const size_t static_bytes = hp.statics.size() * sizeof(float) + aabb.size() * sizeof(float) +
                              static_bs.size() * sizeof(float) + slot_bs.size() * sizeof(float) +
                              group_bs.size() * sizeof(float) + gm_bytes + ms_bytes;
  size_t o_st = section(static_bytes);
  size_t o_sty = section(hp.static_type.size() * sizeof(int));
  size_t o_ti = section(tiles.size() * sizeof(TileInfo));
  size_t o_en = section(entries.size() * sizeof(TileEntry));
  size_t o_ge = section(generic.size() * sizeof(GenericPair));
  size_t o_sg = section(segs.size() * sizeof(GenSeg));
  size_t o_ru = section(runs.size() * sizeof(PairRun));
  size_t o_status = section(16);
  size_t o_ls = section(link_slot.size() * sizeof(int));
  size_t o_lf = section(link_fixed.size() * sizeof(float));
  std::vector<char> host_blob(off, 0);
  auto put = [&](size_t o, const void* src, size_t n) {
    if (n) std::memcpy(host_blob.data() + o, src, n);
  };
  put(o_fk, fk.data(), fk.size() * sizeof(FkJoint));
  put(o_mv, hp.moving.data(), hp.moving.size() * sizeof(MovingGeom));
  put(o_st, hp.statics.data(), hp.statics.size() * sizeof(float));
  put(o_st + hp.statics.size() * sizeof(float), aabb.data(), aabb.size() * sizeof(float));
  const size_t o_sph = o_st + (hp.statics.size() + aabb.size()) * sizeof(float);
  const size_t o_slb = o_sph + static_bs.size() * sizeof(float);
  const size_t o_gbs = o_slb + slot_bs.size() * sizeof(float);
  const size_t o_gmk = o_gbs + group_bs.size() * sizeof(float);
  const size_t o_msl = o_gmk + gm_bytes;
  put(o_sph, static_bs.data(), static_bs.size() * sizeof(float));
  put(o_slb, slot_bs.data(), slot_bs.size() * sizeof(float));
  put(o_gbs, group_bs.data(), group_bs.size() * sizeof(float));
  put(o_gmk, group_mask.data(), group_mask.size() * sizeof(uint32_t));
  put(o_msl, moving_slot.data(), moving_slot.size());
  put(o_sty, hp.static_type.data(), hp.static_type.size() * sizeof(int));
  put(o_ti, tiles.data(), tiles.size() * sizeof(TileInfo));
  put(o_en, entries.data(), entries.size() * sizeof(TileEntry));
  put(o_ge, generic.data(), generic.size() * sizeof(GenericPair));
  put(o_sg, segs.data(), segs.size() * sizeof(GenSeg));
  put(o_ru, runs.data(), runs.size() * sizeof(PairRun));
  put(o_ls, link_slot.data(), link_slot.size() * sizeof(int));
  put(o_lf, link_fixed.data(), link_fixed.size() * sizeof(float));
  CSD_CUDA_TRY(cudaMalloc(&h->blob, off));
  CSD_CUDA_TRY(cudaMemcpy(h->blob, host_blob.data(), off, cudaMemcpyHostToDevice));
  char* base = (char*)h->blob;
  DevPlant& dp = h->dp;
  dp.dim = D;
  dp.num_fk = (int)fk.size();
  dp.num_slots = (int)fk.size();
  dp.num_moving = (int)hp.moving.size();
  dp.num_msph = nmsph;
  dp.num_mcap = (int)mov_cap.size();
  dp.num_tiles = T;
  dp.num_static = S;
  dp.num_ssph = (int)st_sph.size();
  dp.num_sabox = (int)st_abox.size();
  dp.num_srbox = (int)st_rbox.size();
  dp.num_scap = (int)st_cap.size();
  dp.num_generic = (int)generic.size();
  dp.num_segs = (int)segs.size();
  dp.static_bytes = (int)static_bytes;
  dp.pose_words = pose_words;
  dp.always_colliding = always;
  {
    int dense = T > 0;
    for (int t = 0; t < T; ++t) dense &= tiles[t].dense[SC_SPH] && tiles[t].dense[SC_ABOX];
    dp.dense_spheres = dense;
  }
  dp.num_links = L;
  dp.cull = NSL >= 1 && NSL <= 32 && S <= 32 * 32;
  h->cull_eligible = dp.cull != 0;
  dp.slot_bs = (const float4*)(base + o_slb);
  dp.moving_slot = (const uint8_t*)(base + o_msl);
  dp.fk = (const FkJoint*)(base + o_fk);
  dp.moving = (const MovingGeom*)(base + o_mv);
  dp.statics = (const float4*)(base + o_st);
  dp.aabb = (const float4*)(base + o_st + hp.statics.size() * sizeof(float));
  dp.static_type = (const int*)(base + o_sty);
  dp.tiles = (const TileInfo*)(base + o_ti);
  dp.entries = (const TileEntry*)(base + o_en);
  dp.generic = (const GenericPair*)(base + o_ge);
  dp.segs = (const GenSeg*)(base + o_sg);
  dp.runs = (const PairRun*)(base + o_ru);
  dp.status = (int*)(base + o_status);
  dp.link_slot = (const int*)(base + o_ls);
  dp.link_fixed = (const float*)(base + o_lf);
  *out = h.release();
  return CSD_OK;
}

csd_status_t csd_plant_destroy(csd_plant_t p) {
  if (!p) return CSD_OK;
  int cur = 0, dev = p->device;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  delete p;
  if (cur != dev) cudaSetDevice(cur);
  return CSD_OK;
}

csd_status_t csd_plant_set_culling(csd_plant_t p, int32_t enable) {
  CSD_CHECK(p, CSD_ERR_INVALID, "null plant");
  p->dp.cull = (enable && p->cull_eligible) ? 1 : 0;
  return CSD_OK;
}

csd_status_t csd_plant_flops(csd_plant_t p, double* fk, double* place, double* pairs) {
  CSD_CHECK(p && fk && place && pairs, CSD_ERR_INVALID, "null argument");
  *fk = p->host.flops_fk;
  *place = p->host.flops_place;
  *pairs = p->host.flops_pairs;
  return CSD_OK;
}

csd_status_t csd_plant_info(csd_plant_t p, csd_plant_info_t* info) {
  CSD_CHECK(p && info, CSD_ERR_INVALID, "null argument");
  info->dim = p->dp.dim;
  info->num_links = p->dp.num_links;
  info->num_fk_joints = p->dp.num_fk;
  info->num_moving = p->dp.num_moving;
  info->num_static = p->dp.num_static;
  info->num_tile_pairs = p->host.num_tile_pairs;
  info->num_generic_pairs = p->dp.num_generic;
  info->always_colliding = p->dp.always_colliding;
  return CSD_OK;
}

}  // extern "C"
