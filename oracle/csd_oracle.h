/*
 * csd_oracle.h -- CPU oracle for the CSDecomp hot path (TEST INFRASTRUCTURE).
 *
 * This library is the checker, never the product: only tests/, the smoke()
 * entry of __graft_entry__.py and the cpu_baseline / reference arms of
 * bench.py may load it. It restates, in plain C++ without Eigen, the
 * reference algorithms cited function by function in csd_oracle.cpp:
 *
 *   forward kinematics      csdecomp/src/plant/minimal_kinematic_tree.cpp:10-58
 *   pair tests (CPU rules)  csdecomp/src/plant/collision_checker.cpp:91-203
 *   pair tests (GPU rules)  csdecomp/src/geometry/cuda_geometry_utilities.h:16-125
 *   point check             csdecomp/src/plant/collision_checker.cpp:9-39,55-89
 *   edge check              csdecomp/src/plant/collision_checker.cpp:41-53
 *                           csdecomp/src/planning/cuda_visibility_graph.cu:58-72,123-172
 *   hit-and-run             csdecomp/src/geometry/cuda_hit_and_run_sampling.cu:18-119
 *   EI-ZO loop              csdecomp/src/planning/cuda_edge_inflation_zero_order.cu:94-339
 *                           csdecomp/src/planning/cuda_set_builder_utils.cu:25-455
 *   region editing          csdecomp/src/planning/cuda_edit_regions.cu:44-301
 *
 * Capsules have no reference semantics (the reference throws on them); the
 * oracle defines them in FP64 as sphere-swept segments along the local z axis.
 *
 * The plant layout below is a flat, pointer-based mirror of the reference's
 * MinimalPlant (csdecomp/src/plant/minimal_plant.h:16-39); the product's C-ABI
 * uses the same field order so a test can hand one set of arrays to both.
 */
#ifndef CSD_ORACLE_H
#define CSD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t num_joints;
  int32_t num_links;
  int32_t num_configuration_variables;
  int32_t num_geometries;
  int32_t num_collision_pairs;
  const int32_t* joint_type;               /* [J] 0 FIXED, 1 REVOLUTE, 2 PRISMATIC */
  const int32_t* joint_parent_link;        /* [J] */
  const int32_t* joint_child_link;         /* [J] */
  const int32_t* joint_idx_to_config_idx;  /* [J] (-1 for fixed joints) */
  const int32_t* joint_traversal_sequence; /* [J] DFS order */
  const float* joint_X_PL_J;               /* [J][16] 4x4 column-major */
  const float* joint_axis;                 /* [J][3] */
  const int32_t* geom_type;                /* [G] 0 BOX, 1 SPHERE, 2 CYLINDER, 3 CAPSULE */
  const int32_t* geom_link_index;          /* [G] */
  const int32_t* geom_group;               /* [G] 0 ROBOT, 1 WORLD, 2 VOXELS */
  const float* geom_dimensions;            /* [G][3] box: full extents; sphere: (r,-1,-1);
                                              capsule: (r, length, r) */
  const float* geom_X_L_B;                 /* [G][16] 4x4 column-major */
  const int32_t* collision_pairs_flat;     /* [2P] a0 b0 a1 b1 ... */
} orc_plant_t;

/* Pair-test contact rules. */
enum { ORC_RULE_CPU = 0, ORC_RULE_GPU = 1 };
/* Edge discretisation rules. */
enum { ORC_EDGE_L2_REF = 0, ORC_EDGE_LINF = 1, ORC_EDGE_VG = 2 };

/* Forward kinematics, FP32 in the reference CPU operation order (no FMA). tf: [N][L][16]. */
int orc_fk_f32(const orc_plant_t* p, const float* q, int64_t n, float* tf);
/* Forward kinematics in FP64 (q given in FP32 and promoted). tf: [N][L][16]. */
int orc_fk_f64(const orc_plant_t* p, const float* q, int64_t n, double* tf);

/* Point check: out[i] = 1 iff config i is collision free. voxels [V][3]. */
int orc_check_points(const orc_plant_t* p, const float* q, int64_t n, int rule,
                     const float* voxels, int32_t num_voxels, float voxel_radius,
                     const int32_t* robot_geom_ids, int32_t num_robot_geoms,
                     uint8_t* out, int nthreads);

/* FP64 signed distances: for each config, the FP64 verdict (1 = free) and the
 * minimum signed distance over all pairs (and voxel pairs) in metres. A
 * config lies in the contact band when |min signed distance| <= 1e-5 m: only
 * then can FP32 rounding flip its verdict. */
int orc_signed_distance_f64(const orc_plant_t* p, const float* q, int64_t n,
                            const float* voxels, int32_t num_voxels, float voxel_radius,
                            const int32_t* robot_geom_ids, int32_t num_robot_geoms,
                            uint8_t* verdict64, double* min_sd, int nthreads);

/* Edge check with early exit. starts/ends: [E][d]. out[e] = 1 iff free. */
int orc_check_edges(const orc_plant_t* p, const float* starts, const float* ends, int64_t e,
                    float step, int mode, int rule, uint8_t* out, int64_t* points_checked,
                    int nthreads);

/* Number of discretisation points of one edge under a rule (for tests). */
int64_t orc_edge_num_points(const float* q1, const float* q2, int32_t dim, float step, int mode);
/* The k-th discretisation point of one edge under a rule. */
void orc_edge_point(const float* q1, const float* q2, int32_t dim, float step, int mode,
                    int64_t k, float* out);

/* Single pair test; X_W_LA, X_W_LB column-major 4x4. Returns 1 if free, 0 if
 * colliding, -1 on unsupported shapes. */
int orc_pair_collision_free(int32_t type_a, const float* dims_a, const float* X_L_B_a,
                            const float* X_W_LA, int32_t type_b, const float* dims_b,
                            const float* X_L_B_b, const float* X_W_LB, int rule);

/* Hit-and-run sampling (the build's Philox4x32-10 stream, see csd_oracle.cpp).
 * A [F][d] row-major, b [F]; samples [S][d]; starts from x0. Chains whose
 * theta-interval is empty are written as NaN and counted in *num_failed. */
int orc_hit_and_run(const float* A, const float* b, int32_t num_faces, int32_t dim,
                    const float* x0, int32_t num_samples, int32_t mixing_steps, uint64_t seed,
                    uint32_t stream, float* samples, int32_t* num_failed, int nthreads);

/* Philox4x32-10 block function (known-answer tests). */
void orc_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out);
/* Gaussian/uniform stream used by the sampler (for bit-exact GPU tests). */
void orc_rng_uniform(uint64_t seed, uint32_t chain, uint32_t stream, uint32_t step, float* out4);
void orc_rng_direction(uint64_t seed, uint32_t chain, uint32_t stream, uint32_t step,
                       int32_t dim, float* dir);

typedef struct {
  float configuration_margin;
  float tau;
  float delta;
  float epsilon;
  uint32_t bisection_steps;
  uint32_t num_particles;
  uint32_t max_hyperplanes_per_iteration;
  uint32_t max_iterations;
  uint32_t mixing_steps;
  uint64_t seed;
} orc_eizo_options_t;

typedef struct {
  int32_t iteration_index;
  int32_t num_samples_drawn;
  int32_t collisions_threshold;
  int32_t num_collisions_unadaptive;
  int32_t num_collisions_updated;
  int32_t num_faces_placed;
} orc_eizo_iter_t;

/* Batch collision checker callback: out[i] = 1 iff q[i] free. Returns 0 on success. */
typedef int (*orc_checker_fn)(const float* q, int64_t n, uint8_t* out, void* ctx);

/* EI-ZO on the CPU. A/b hold the domain on entry (num_faces rows) and the
 * region on exit; capacity = rows available in A/b. If checker is NULL the
 * oracle's own point check (GPU contact rule) is used. iters may be NULL.
 * Returns 0 on success, 2 on face capacity exceeded. */
int orc_eizo(const orc_plant_t* p, const float* line_start, const float* line_end,
             const float* voxels, int32_t num_voxels, float voxel_radius,
             const int32_t* robot_geom_ids, int32_t num_robot_geoms,
             const orc_eizo_options_t* opt, float* A, float* b, int32_t* num_faces,
             int32_t capacity, orc_checker_fn checker, void* checker_ctx,
             orc_eizo_iter_t* iters, int32_t* num_iters, int nthreads);

/* numSamplesUnadaptive, csdecomp/src/planning/cuda_set_builder_utils.h:198-203 */
uint32_t orc_num_samples_unadaptive(float epsilon, float delta, float tau);

/* EditRegionsCuda, csdecomp/src/planning/cuda_edit_regions.cu:44-301.
 * collisions [n][d] with their segment indices; starts/ends [m][d]; region r
 * is rows [face_offsets[r], face_offsets[r+1]) of A (row-major) and b. Region
 * r comes back at row face_offsets[r] + (collisions of segments < r) of
 * A_out/b_out with num_faces[r] rows; proj_out/opt_out are [n][d] in the
 * grouped (segment-stable) order. checker (may be NULL) replaces the
 * oracle's own point check. Returns 0, -1 dim > 16, -2 segment index out of
 * range, -3 point check failed. */
int orc_edit_regions(const orc_plant_t* p, const float* collisions, const uint32_t* seg, int64_t n,
                     const float* starts, const float* ends, int32_t m, const float* A, const float* b,
                     const int32_t* face_offsets, const float* voxels, int32_t nv, float vr,
                     const int32_t* robot_geom_ids, int32_t num_robot_geoms, float margin,
                     uint32_t bisection_steps, float* A_out, float* b_out, int32_t* num_faces,
                     float* proj_out, float* opt_out, orc_checker_fn checker, void* checker_ctx,
                     int nthreads);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
