/*
 * csd_cpp.hpp -- header-only C++ adapter: the reference's C++ host API for the
 * hot path, over the C ABI of csd_capi.h. It needs no Eigen and no reference
 * headers: the reference's types enter as template parameters and are read by
 * the reference's member names, so the reference's own
 *   csdecomp::MinimalPlant / MinimalKinematicTree (minimal_plant.h:16-39,
 *   minimal_kinematic_tree.h:18-53), Eigen::MatrixXf / VectorXf, Voxels
 *   (collision_geometry.h:63) and EizoOptions (cuda_edge_inflation_zero_order.h:18-32)
 * instantiate it directly. Matrices are read through rows(), cols() and
 * data() (column major, as Eigen's default); 4x4 transforms and 3-vectors
 * through operator()(row, col) and operator()(i).
 *
 * Errors: CSD_ERR_INVALID is rethrown as std::invalid_argument, every other
 * failure as std::runtime_error (the reference's exception types), with the
 * library's message. Calls synchronise their stream before returning, as the
 * reference's functions do.
 */
#ifndef CSD_CPP_HPP
#define CSD_CPP_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "csd_capi.h"

namespace csd_cpp {

inline void check(csd_status_t s) {
  if (s == CSD_OK) return;
  const char* m = csd_last_error();
  const std::string msg = m ? m : "csdecomp_b200 error";
  if (s == CSD_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

/* A plant uploaded once to the current device (csd_plant_create). The
 * reference uploads its ~270 KB MinimalPlant on every call
 * (cuda_collision_checker.cu:458-462); here a DevicePlant is made once and
 * reused. Move-only. */
class DevicePlant {
 public:
  DevicePlant() = default;
  explicit DevicePlant(const csd_plant_desc_t& desc) { check(csd_plant_create(&desc, &h_)); }
  DevicePlant(const DevicePlant&) = delete;
  DevicePlant& operator=(const DevicePlant&) = delete;
  DevicePlant(DevicePlant&& o) noexcept : h_(o.h_), dim_(o.dim_), links_(o.links_) { o.h_ = nullptr; }
  DevicePlant& operator=(DevicePlant&& o) noexcept {
    std::swap(h_, o.h_);
    std::swap(dim_, o.dim_);
    std::swap(links_, o.links_);
    return *this;
  }
  ~DevicePlant() {
    if (h_) csd_plant_destroy(h_);
  }
  csd_plant_t get() const { return h_; }
  int dim() const { return dim_; }
  int num_links() const { return links_; }

 private:
  template <class P>
  friend DevicePlant upload(const P& mp);
  csd_plant_t h_ = nullptr;
  int dim_ = 0, links_ = 0;
};

/* Flattens a MinimalPlant (any type with the reference's members) into the
 * ABI's tables and uploads it. Joint and geometry enums map by value (FIXED,
 * REVOLUTE, PRISMATIC = 0, 1, 2; BOX, SPHERE, CYLINDER, CAPSULE = 0..3;
 * ROBOT, WORLD, VOXELS = 0..2), as in the reference. */
template <class P>
DevicePlant upload(const P& mp) {
  const auto& kt = mp.kin_tree;
  const int J = kt.num_joints, G = mp.num_scene_geometries, NP = mp.num_collision_pairs;
  std::vector<int32_t> jt(J), jp(J), jc(J), jq(J), js(J), gt(G), gl(G), gg(G), pairs(2 * (size_t)NP);
  std::vector<float> X(16 * (size_t)J), ax(3 * (size_t)J), gd(3 * (size_t)G), XB(16 * (size_t)G);
  for (int j = 0; j < J; ++j) {
    const auto& jn = kt.joints[j];
    jt[j] = (int32_t)jn.type;
    jp[j] = jn.parent_link;
    jc[j] = jn.child_link;
    jq[j] = kt.joint_idx_to_config_idx[j];
    js[j] = kt.joint_traversal_sequence[j];
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) X[16 * (size_t)j + 4 * c + r] = jn.X_PL_J(r, c);
    for (int k = 0; k < 3; ++k) ax[3 * (size_t)j + k] = jn.axis(k);
  }
  for (int g = 0; g < G; ++g) {
    const auto& cg = mp.scene_collision_geometries[g];
    gt[g] = (int32_t)cg.type;
    gl[g] = cg.link_index;
    gg[g] = (int32_t)cg.group;
    for (int k = 0; k < 3; ++k) gd[3 * (size_t)g + k] = cg.dimensions(k);
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) XB[16 * (size_t)g + 4 * c + r] = cg.X_L_B(r, c);
  }
  for (int i = 0; i < 2 * NP; ++i) pairs[i] = mp.collision_pairs_flat[i];
  csd_plant_desc_t d{};
  d.num_joints = J;
  d.num_links = kt.num_links;
  d.num_configuration_variables = kt.num_configuration_variables;
  d.num_geometries = G;
  d.num_collision_pairs = NP;
  d.joint_type = jt.data();
  d.joint_parent_link = jp.data();
  d.joint_child_link = jc.data();
  d.joint_idx_to_config_idx = jq.data();
  d.joint_traversal_sequence = js.data();
  d.joint_X_PL_J = X.data();
  d.joint_axis = ax.data();
  d.geom_type = gt.data();
  d.geom_link_index = gl.data();
  d.geom_group = gg.data();
  d.geom_dimensions = gd.data();
  d.geom_X_L_B = XB.data();
  d.collision_pairs_flat = pairs.data();
  DevicePlant out(d);
  out.dim_ = d.num_configuration_variables;
  out.links_ = d.num_links;
  return out;
}

/* checkCollisionFreeCuda (cuda_collision_checker.h:93-94): q is dim x N,
 * column major; one byte per configuration, 1 = collision free. */
template <class M>
std::vector<uint8_t> checkCollisionFreeCuda(const M* q, const DevicePlant& plant) {
  if (q->rows() != plant.dim()) throw std::runtime_error("configuration dimension does not match the plant");
  std::vector<uint8_t> out((size_t)q->cols());
  check(csd_check_points(plant.get(), q->data(), (int64_t)q->cols(), nullptr, 0, 0.f, nullptr, 0, out.data(),
                         CSD_PTR_HOST, nullptr));
  return out;
}
/* The reference's exact signature: uploads the plant for this call. */
template <class M, class P>
std::vector<uint8_t> checkCollisionFreeCuda(const M* q, const P* mp) {
  return checkCollisionFreeCuda(q, upload(*mp));
}

/* checkCollisionFreeVoxelsCuda (cuda_collision_checker.h:112-115): voxels is
 * 3 x V, column major. */
template <class M, class V>
std::vector<uint8_t> checkCollisionFreeVoxelsCuda(const M* q, const V* voxels, float voxel_radius,
                                                  const DevicePlant& plant,
                                                  const std::vector<int32_t>& robot_geometry_ids) {
  if (q->rows() != plant.dim()) throw std::runtime_error("configuration dimension does not match the plant");
  std::vector<uint8_t> out((size_t)q->cols());
  check(csd_check_points(plant.get(), q->data(), (int64_t)q->cols(), voxels->data(), (int32_t)voxels->cols(),
                         voxel_radius, robot_geometry_ids.data(), (int32_t)robot_geometry_ids.size(), out.data(),
                         CSD_PTR_HOST, nullptr));
  return out;
}

/* computeForwardKinematicsCuda (cuda_forward_kinematics.h:53-55): transforms
 * receives [N][num_links][16] column-major 4x4s, i.e. a 16 x (N num_links)
 * column-major matrix (resized here through resize(rows, cols)). */
template <class M>
void computeForwardKinematicsCuda(M* transforms, const M* q, const DevicePlant& plant) {
  if (q->rows() != plant.dim()) throw std::runtime_error("configuration dimension does not match the plant");
  transforms->resize(16, q->cols() * plant.num_links());
  check(csd_fk(plant.get(), q->data(), (int64_t)q->cols(), transforms->data(), CSD_PTR_HOST, nullptr));
}

/* Batched edge checks with early exit (new): starts/ends dim x E; mode one of
 * CSD_EDGE_L2_REF (checkEdgeCollisionFree's rule, collision_checker.cpp:41-53),
 * CSD_EDGE_LINF, CSD_EDGE_VG. */
template <class M>
std::vector<uint8_t> checkEdgesCollisionFreeCuda(const M* starts, const M* ends, const DevicePlant& plant,
                                                 float step_size = 0.01f, int32_t mode = CSD_EDGE_L2_REF) {
  if (starts->rows() != plant.dim() || ends->rows() != plant.dim() || starts->cols() != ends->cols())
    throw std::runtime_error("edge endpoints must be dim x E each");
  std::vector<uint8_t> out((size_t)starts->cols());
  check(csd_check_edges(plant.get(), starts->data(), ends->data(), (int64_t)starts->cols(), step_size, mode,
                        out.data(), nullptr, CSD_PTR_HOST, nullptr));
  return out;
}

/* An H-polytope {x : A x <= b} as the library returns it: A row major. */
struct Region {
  int dim = 0;
  std::vector<float> A, b;
  int num_faces() const { return (int)b.size(); }
};

/* EizoOptions (cuda_edge_inflation_zero_order.h:18-32) to the ABI struct. */
template <class O>
csd_eizo_options_t eizo_options(const O& o) {
  csd_eizo_options_t c{};
  c.configuration_margin = o.configuration_margin;
  c.tau = o.tau;
  c.delta = o.delta;
  c.epsilon = o.epsilon;
  c.bisection_steps = o.bisection_steps;
  c.num_particles = o.num_particles;
  c.max_hyperplanes_per_iteration = o.max_hyperplanes_per_iteration;
  c.max_iterations = o.max_iterations;
  c.mixing_steps = o.mixing_steps;
  c.seed = o.seed;
  c.verbose = o.verbose ? 1 : 0;
  c.track_iteration_information = o.track_iteration_information ? 1 : 0;
  return c;
}

/* CudaEdgeInflator (cuda_polytope_builder.h:16-44): built once per plant,
 * options and domain; inflateEdge grows a region around a collision-free
 * segment. The domain is given as A (F x dim, column major, as Eigen) and b. */
class CudaEdgeInflator {
 public:
  template <class P, class O, class MA, class VB>
  CudaEdgeInflator(const P& plant, const std::vector<int32_t>& robot_geometry_ids, const O& options,
                   const MA& domain_A, const VB& domain_b, int max_voxels = 10000, int face_capacity = 4000)
      : plant_(upload(plant)), dim_(plant_.dim()) {
    const int F = (int)domain_A.rows();
    if (domain_A.cols() != dim_ || domain_b.size() != F) throw std::runtime_error("domain must be F x dim and F");
    std::vector<float> A((size_t)F * dim_), b(F);
    for (int f = 0; f < F; ++f) {
      for (int k = 0; k < dim_; ++k) A[(size_t)f * dim_ + k] = domain_A(f, k);
      b[f] = domain_b(f);
    }
    const csd_eizo_options_t o = eizo_options(options);
    check(csd_inflator_create(plant_.get(), robot_geometry_ids.data(), (int32_t)robot_geometry_ids.size(), &o,
                              A.data(), b.data(), F, max_voxels, face_capacity, &h_));
    capacity_ = face_capacity;
  }
  CudaEdgeInflator(const CudaEdgeInflator&) = delete;
  CudaEdgeInflator& operator=(const CudaEdgeInflator&) = delete;
  ~CudaEdgeInflator() {
    if (h_) csd_inflator_destroy(h_);
  }
  /* voxels: 3 x V column major (may be empty). */
  template <class VEC, class V>
  Region inflateEdge(const VEC& line_start, const VEC& line_end, const V& voxels, float voxel_radius,
                     bool verbose = true) {
    (void)verbose;  // the library reports per-iteration information through csd_inflator_inflate's info array
    if ((int)line_start.size() != dim_ || (int)line_end.size() != dim_)
      throw std::runtime_error("segment dimension does not match the plant");
    Region r;
    r.dim = dim_;
    r.A.resize((size_t)capacity_ * dim_);
    r.b.resize(capacity_);
    int32_t nf = 0;
    check(csd_inflator_inflate(h_, line_start.data(), line_end.data(), voxels.cols() ? voxels.data() : nullptr,
                               (int32_t)voxels.cols(), voxel_radius, r.A.data(), r.b.data(), &nf, nullptr, 0, nullptr,
                               nullptr));
    r.A.resize((size_t)nf * dim_);
    r.b.resize(nf);
    return r;
  }

 private:
  DevicePlant plant_;
  int dim_ = 0, capacity_ = 0;
  csd_inflator_t h_ = nullptr;
};

/* UniformSampleInHPolyhedronCuda (cuda_hit_and_run_sampling.h:25-52) for one
 * polytope: num_samples points (num_samples x dim, row major), NaN rows for
 * chains whose line search failed. */
inline std::vector<float> uniformSampleInHPolyhedronCuda(const Region& poly, const std::vector<float>& start,
                                                         int num_samples, int mixing_steps, uint64_t seed = 1337) {
  std::vector<float> out((size_t)num_samples * poly.dim);
  const int32_t off[2] = {0, poly.num_faces()};
  int32_t failed = 0;
  check(csd_uniform_sample_hpolyhedra(poly.A.data(), poly.b.data(), off, 1, poly.dim, start.data(), num_samples,
                                      mixing_steps, seed, out.data(), &failed, CSD_PTR_HOST, nullptr));
  return out;
}

}  // namespace csd_cpp

#endif  // CSD_CPP_HPP
