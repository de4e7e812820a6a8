// Compiles include/csd_cpp.hpp against stand-ins of the reference's types
// (member names of minimal_plant.h, minimal_kinematic_tree.h,
// collision_geometry.h, cuda_edge_inflation_zero_order.h; a column-major
// matrix with Eigen's accessors) and exercises it on a one-joint arm:
// a revolute joint about z at the origin carries a sphere of radius 0.1 at
// x = 1.2; a world box of full extents 1 x 1 x 1 is centred at (1.5, 0, 0).
// q = 0 puts the sphere inside the box, q = pi puts it 2.7 m away.
//   adapter_demo nodevice : without a GPU, the upload must throw std::runtime_error
//   adapter_demo device   : checks, FK, edges, EI-ZO and sampling on the GPU
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "csd_cpp.hpp"

namespace ref {  // stand-ins with the reference's member names
struct Matrix4f {
  float m[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};  // column major
  float operator()(int r, int c) const { return m[4 * c + r]; }
  float& operator()(int r, int c) { return m[4 * c + r]; }
};
struct Vector3f {
  float v[3] = {0, 0, 0};
  float operator()(int i) const { return v[i]; }
};
struct MatrixXf {  // column major, as Eigen::MatrixXf
  int r = 0, c = 0;
  std::vector<float> d;
  MatrixXf(int rows = 0, int cols = 0) : r(rows), c(cols), d((size_t)rows * cols) {}
  int rows() const { return r; }
  int cols() const { return c; }
  int size() const { return r * c; }
  const float* data() const { return d.data(); }
  float* data() { return d.data(); }
  void resize(int rows, int cols) { r = rows, c = cols, d.assign((size_t)rows * cols, 0.f); }
  float operator()(int i, int j) const { return d[(size_t)j * r + i]; }
  float& operator()(int i, int j) { return d[(size_t)j * r + i]; }
  float operator()(int i) const { return d[i]; }
};
enum JointType { FIXED, REVOLUTE, PRISMATIC };
enum ShapePrimitive { BOX, SPHERE, CYLINDER, CAPSULE };
enum CollisionGroup { ROBOT, WORLD, VOXELS };
struct MinimalJoint {
  JointType type;
  Matrix4f X_PL_J;
  int index, parent_link, child_link;
  Vector3f axis;
};
struct MinimalKinematicTree {
  MinimalJoint joints[4];
  int joint_traversal_sequence[4];
  int joint_idx_to_config_idx[4];
  int num_configuration_variables, num_joints, num_links;
};
struct CollisionGeometry {
  ShapePrimitive type;
  Vector3f dimensions;
  int link_index;
  CollisionGroup group;
  Matrix4f X_L_B;
};
struct MinimalPlant {
  MinimalKinematicTree kin_tree;
  CollisionGeometry scene_collision_geometries[4];
  int32_t collision_pairs_flat[8];
  int32_t num_scene_geometries, num_collision_pairs;
};
struct EizoOptions {
  float configuration_margin = 0.01f, tau = 0.5f, delta = 0.05f, epsilon = 0.01f;
  unsigned bisection_steps = 9, num_particles = 400, max_hyperplanes_per_iteration = 10, max_iterations = 50,
           mixing_steps = 20;
  uint64_t seed = 1337;
  bool verbose = false, track_iteration_information = false;
};
}  // namespace ref

static ref::MinimalPlant one_joint_arm() {
  ref::MinimalPlant p{};
  auto& kt = p.kin_tree;
  kt.num_links = 3;  // world (0), arm link (1), obstacle carrier (2)
  kt.num_joints = 2;
  kt.num_configuration_variables = 1;
  kt.joints[0] = {ref::REVOLUTE, {}, 0, 0, 1, {{0, 0, 1}}};
  kt.joints[1] = {ref::FIXED, {}, 1, 0, 2, {{0, 0, 1}}};
  kt.joint_traversal_sequence[0] = 0;
  kt.joint_traversal_sequence[1] = 1;
  kt.joint_idx_to_config_idx[0] = 0;
  kt.joint_idx_to_config_idx[1] = -1;
  auto& s = p.scene_collision_geometries[0];
  s = {ref::SPHERE, {{0.1f, -1.f, -1.f}}, 1, ref::ROBOT, {}};
  s.X_L_B(0, 3) = 1.2f;
  auto& b = p.scene_collision_geometries[1];
  b = {ref::BOX, {{1.f, 1.f, 1.f}}, 2, ref::WORLD, {}};
  b.X_L_B(0, 3) = 1.5f;
  p.num_scene_geometries = 2;
  p.collision_pairs_flat[0] = 0;
  p.collision_pairs_flat[1] = 1;
  p.num_collision_pairs = 1;
  return p;
}

#define REQUIRE(c)                                                  \
  do {                                                              \
    if (!(c)) {                                                     \
      std::fprintf(stderr, "failed: %s (line %d)\n", #c, __LINE__); \
      return 1;                                                     \
    }                                                               \
  } while (0)

int main(int argc, char** argv) {
  const bool device = argc > 1 && std::strcmp(argv[1], "device") == 0;
  const ref::MinimalPlant mp = one_joint_arm();
  int32_t nsv = 0, ncc = 0;
  csd_batch_shape_counts(&nsv, &ncc);  // needs no device
  REQUIRE(nsv > 0 && ncc > 0);
  if (!device) {
    try {
      csd_cpp::DevicePlant p = csd_cpp::upload(mp);
      std::fprintf(stderr, "upload succeeded without a device\n");
      return 1;
    } catch (const std::runtime_error& e) {
      std::printf("no device: %s\n", e.what());
    }
    try {
      csd_cpp::check(CSD_ERR_INVALID);
      return 1;
    } catch (const std::invalid_argument&) {
    }
    std::printf("ok\n");
    return 0;
  }
  const csd_cpp::DevicePlant plant = csd_cpp::upload(mp);
  REQUIRE(plant.dim() == 1 && plant.num_links() == 3);
  ref::MatrixXf q(1, 4);
  q(0, 0) = 0.f;
  q(0, 1) = 3.14159f;
  q(0, 2) = -3.14159f;
  q(0, 3) = 0.05f;
  const std::vector<uint8_t> v = csd_cpp::checkCollisionFreeCuda(&q, plant);
  REQUIRE(v.size() == 4 && v[0] == 0 && v[1] == 1 && v[2] == 1 && v[3] == 0);
  REQUIRE(csd_cpp::checkCollisionFreeCuda(&q, &mp) == v);  // the reference's signature (upload per call)
  ref::MatrixXf tf;
  csd_cpp::computeForwardKinematicsCuda(&tf, &q, plant);
  REQUIRE(tf.rows() == 16 && tf.cols() == 12);
  // link 1 at q = pi: x axis rotated to -x (column 0 of the 4x4: cos, sin, 0, 0)
  REQUIRE(std::fabs(tf(0, 1 * 3 + 1) + 1.f) < 1e-5f);
  ref::MatrixXf s(1, 2), e(1, 2);
  s(0, 0) = 2.5f, e(0, 0) = 3.0f;   // free edge
  s(0, 1) = 2.5f, e(0, 1) = -0.5f;  // crosses q = 0
  const std::vector<uint8_t> ev = csd_cpp::checkEdgesCollisionFreeCuda(&s, &e, plant);
  REQUIRE(ev.size() == 2 && ev[0] == 1 && ev[1] == 0);
  ref::MatrixXf dA(2, 1), db(2, 1);
  dA(0, 0) = -1.f, dA(1, 0) = 1.f, db(0, 0) = 3.14159f, db(1, 0) = 3.14159f;
  ref::EizoOptions opt;
  csd_cpp::CudaEdgeInflator inf(mp, {0}, opt, dA, db);
  ref::MatrixXf ls(1, 1), le(1, 1), vox(3, 0);
  ls(0, 0) = 2.5f, le(0, 0) = 3.0f;
  const csd_cpp::Region r = inf.inflateEdge(ls, le, vox, 0.f, false);
  REQUIRE(r.dim == 1 && r.num_faces() >= 2);
  for (float x : {2.5f, 3.0f}) {
    for (int f = 0; f < r.num_faces(); ++f) REQUIRE(r.A[f] * x <= r.b[f] + 1e-6f);
  }
  // the region excludes q = 0 (the sphere inside the box)
  bool excluded = false;
  for (int f = 0; f < r.num_faces(); ++f) excluded |= r.A[f] * 0.f > r.b[f];
  REQUIRE(excluded);
  const std::vector<float> smp = csd_cpp::uniformSampleInHPolyhedronCuda(r, {2.75f}, 64, 10);
  for (float x : smp)
    for (int f = 0; f < r.num_faces(); ++f) REQUIRE(r.A[f] * x <= r.b[f] + 1e-5f);
  std::printf("ok faces=%d\n", r.num_faces());
  return 0;
}
