/*
 * csd_capi.h -- C ABI of csdecomp_b200, the B200 (sm_100a) implementation of
 * CSDecomp's hot path: batched forward kinematics, primitive-pair collision
 * checking over a MinimalPlant, batched edge checks, hit-and-run sampling in
 * an H-polytope, EI-ZO edge inflation, the visibility graph and region
 * editing.
 *
 * Every entry point names the reference interface it replaces (paths are
 * relative to the wernerpe/csdecomp source tree). Conventions:
 *   - configurations are [N][dim] float32, contiguous (= Eigen's column-major
 *     dim x N matrix of the reference);
 *   - transforms are [N][num_links][16] float32, each 4x4 column-major;
 *   - verdicts are uint8, 1 = collision free (the reference's convention);
 *   - polytopes are A [F][dim] row-major float32 and b [F] float32;
 *   - `flags` selects host (CSD_PTR_HOST) or device (CSD_PTR_DEVICE) memory
 *     for the array arguments of a call. Device-pointer calls are ordered on
 *     `stream` (a cudaStream_t, NULL = legacy default stream) and return
 *     without synchronising; host-pointer calls copy through the handle's
 *     device buffers and synchronise `stream` before returning;
 *   - every function returns a csd_status_t; csd_last_error() gives the
 *     message of the last failure on the calling thread. Nothing calls exit().
 * Handles are not thread safe: use one handle per thread or lock externally.
 */
#ifndef CSD_CAPI_H
#define CSD_CAPI_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t csd_status_t;
enum {
  CSD_OK = 0,
  CSD_ERR_INVALID = 1,       /* bad argument (reference: std::invalid_argument / assert) */
  CSD_ERR_CAPACITY = 2,      /* a capacity is exceeded (reference: std::runtime_error) */
  CSD_ERR_NOT_CONTAINED = 3, /* start point outside its polytope (cuda_hit_and_run_sampling.cu:159-164) */
  CSD_ERR_CUDA = 4,          /* CUDA runtime error (reference: CUDACHECKERROR -> exit) */
  CSD_ERR_UNSUPPORTED = 5,   /* cylinders (collision_checker.cpp:104-107) */
  CSD_ERR_DIMENSION = 6,     /* dimension mismatch (reference: std::runtime_error) */
  CSD_ERR_NO_DEVICE = 7      /* no CUDA device visible */
};

enum { CSD_PTR_HOST = 0, CSD_PTR_DEVICE = 1 };

/* Edge discretisation rules for csd_check_edges. */
enum {
  CSD_EDGE_L2_REF = 0, /* T = ceil(|q2-q1|_2 / step), t = k/T, k = 0..T-1 (end excluded):
                          checkEdgeCollisionFree, csdecomp/src/plant/collision_checker.cpp:41-53 */
  CSD_EDGE_LINF = 1,   /* T = ceil(|q2-q1|_inf / step), t = k/T, k = 0..T (both ends) */
  CSD_EDGE_VG = 2      /* n = (uint)(|q2-q1|_2/step + 2) points incl. both ends:
                          csdecomp/src/planning/cuda_visibility_graph.cu:58-72,123-172 */
};

/* Flat view of a MinimalPlant (csdecomp/src/plant/minimal_plant.h:16-39,
 * minimal_kinematic_tree.h:18-53, collision_geometry.h:27-35), with no fixed
 * capacities. All pointers are host memory and are only read during
 * csd_plant_create. */
typedef struct {
  int32_t num_joints;
  int32_t num_links;
  int32_t num_configuration_variables;
  int32_t num_geometries;
  int32_t num_collision_pairs;
  const int32_t* joint_type;               /* [J] 0 FIXED, 1 REVOLUTE, 2 PRISMATIC */
  const int32_t* joint_parent_link;        /* [J] */
  const int32_t* joint_child_link;         /* [J] */
  const int32_t* joint_idx_to_config_idx;  /* [J], -1 for fixed joints */
  const int32_t* joint_traversal_sequence; /* [J] */
  const float* joint_X_PL_J;               /* [J][16] column-major */
  const float* joint_axis;                 /* [J][3] */
  const int32_t* geom_type;                /* [G] 0 BOX, 1 SPHERE, 2 CYLINDER, 3 CAPSULE */
  const int32_t* geom_link_index;          /* [G] */
  const int32_t* geom_group;               /* [G] 0 ROBOT, 1 WORLD, 2 VOXELS */
  const float* geom_dimensions;            /* [G][3] box: full extents; sphere: (r,-1,-1);
                                              capsule: (r, length, r), axis = local z */
  const float* geom_X_L_B;                 /* [G][16] column-major */
  const int32_t* collision_pairs_flat;     /* [2P] */
} csd_plant_desc_t;

typedef struct {
  int32_t dim;             /* configuration variables */
  int32_t num_links;
  int32_t num_fk_joints;   /* moving joints evaluated per configuration */
  int32_t num_moving;      /* geometries whose pose depends on q */
  int32_t num_static;      /* geometries fixed in the world */
  int32_t num_tile_pairs;  /* moving-sphere/static pairs swept by tiles */
  int32_t num_generic_pairs;
  int32_t always_colliding;/* a pair of static geometries collides */
} csd_plant_info_t;

typedef struct csd_plant_s* csd_plant_t;
typedef struct csd_inflator_s* csd_inflator_t;

const char* csd_last_error(void);
int32_t csd_version(void);

/* Native model loader: URDFParser, csdecomp/src/plant/urdf_parser.h:18-163
 * (parseURDF :33, parseURDFString :49, registerPackage :56, parseDirectives
 * :78, getMinimalPlant :86, getSceneInspector().robot_geometry_ids, the
 * kinematic tree's position limits). A handle holds one model. Parse errors
 * (the reference's std::runtime_error, and a root element other than
 * <robot>, for which the reference returns false) give CSD_ERR_INVALID with
 * the message in csd_last_error(). No device is used. */
typedef struct csd_urdf_s* csd_urdf_t;
csd_status_t csd_urdf_create(csd_urdf_t* out);
csd_status_t csd_urdf_destroy(csd_urdf_t h);
/* registered (optional) = 0 when name or path is empty or path does not exist. */
csd_status_t csd_urdf_register_package(csd_urdf_t h, const char* name, const char* path, int32_t* registered);
csd_status_t csd_urdf_parse_file(csd_urdf_t h, const char* path);
csd_status_t csd_urdf_parse_string(csd_urdf_t h, const char* urdf_text);
/* Model directives (add_model, add_weld, add_frame; package:// paths). */
csd_status_t csd_urdf_parse_directives(csd_urdf_t h, const char* path);
/* The parsed MinimalPlant; the pointers stay valid until csd_urdf_destroy and
 * can be passed straight to csd_plant_create. */
csd_status_t csd_urdf_plant_desc(csd_urdf_t h, csd_plant_desc_t* desc);
/* lower/upper: num_configuration_variables floats each. */
csd_status_t csd_urdf_limits(csd_urdf_t h, float* lower, float* upper);
/* Geometries of the ROBOT group (pointer owned by the handle). */
csd_status_t csd_urdf_robot_geometry_ids(csd_urdf_t h, const int32_t** ids, int32_t* n);
csd_status_t csd_urdf_link_index(csd_urdf_t h, const char* name, int32_t* index);
/* scene_collision_geometry_name_to_geometry_index ("<collision name>::<k>" or
 * "<link>::col_geom::<k>", k counting the link's collisions from 1). */
csd_status_t csd_urdf_geometry_index(csd_urdf_t h, const char* name, int32_t* index);

/* Uploads a plant once (device-resident, reusable across calls). Replaces the
 * per-call CudaPtr<const MinimalPlant> upload of checkCollisionFreeCuda,
 * csdecomp/src/plant/cuda_collision_checker.cu:458-462. Uses the current device. */
csd_status_t csd_plant_create(const csd_plant_desc_t* desc, csd_plant_t* out);
csd_status_t csd_plant_destroy(csd_plant_t plant);
csd_status_t csd_plant_info(csd_plant_t plant, csd_plant_info_t* info);

/* Bounded waits: each check kernel stages the plant's static tables into
 * shared memory behind an mbarrier whose wait gives up after a bounded number
 * of polls; the block then returns without checking its configurations and
 * sets the plant's status word. Host-pointer calls (and csd_eizo,
 * csd_inflator_inflate, csd_batch_inflate, csd_edit_regions) read and clear it
 * before returning and fail with CSD_ERR_CUDA; device-pointer callers query
 * it here after their stream's work (timed_out = 1: results since the last
 * query are incomplete). Synchronises `stream`. */
csd_status_t csd_plant_status(csd_plant_t plant, int32_t* timed_out, void* stream);
/* Self-test of that path (no fault, no hang): one block polls `polls` times an
 * mbarrier that nothing completes, gives up as the staging does and sets the
 * status word; reported = 1 when the host read it back (and cleared it). */
csd_status_t csd_plant_wait_selftest(csd_plant_t plant, int32_t polls, int32_t* reported);

/* Forward kinematics: computeForwardKinematicsCuda,
 * csdecomp/src/plant/cuda_forward_kinematics.cu:92-129 (device-pointer form:
 * executeForwardKinematicsKernel, :79-90). transforms: [n][num_links][16]. */
csd_status_t csd_fk(csd_plant_t plant, const float* q, int64_t n, float* transforms, int32_t flags,
                    void* stream);

/* Point check: checkCollisionFreeCuda, csdecomp/src/plant/cuda_collision_checker.cu:437-487,
 * and with voxels (num_voxels > 0) checkCollisionFreeVoxelsCuda, :374-435
 * (device-pointer forms: executeCollisionFreeKernel :182-209,
 * executeCollisionFreeVoxelsKernel :256-307). voxels: [V][3] world positions of
 * voxel spheres of radius voxel_radius, checked against robot_geometry_ids
 * (always host memory, whatever `flags` says; a device pointer is refused). */
csd_status_t csd_check_points(csd_plant_t plant, const float* q, int64_t n, const float* voxels,
                              int32_t num_voxels, float voxel_radius, const int32_t* robot_geometry_ids,
                              int32_t num_robot_geometries, uint8_t* free_out, int32_t flags, void* stream);

/* Batched edge check with early exit (new; the reference's CPU
 * checkEdgeCollisionFree, collision_checker.cpp:41-53, checks one edge; its GPU
 * edge checks live inside VisibilityGraph, cuda_visibility_graph.cu:175-375).
 * starts/ends: [n][dim]. points_checked (optional, [n] int64): points
 * evaluated before the verdict was known. */
csd_status_t csd_check_edges(csd_plant_t plant, const float* starts, const float* ends, int64_t n,
                             float step_size, int32_t mode, uint8_t* free_out, int64_t* points_checked,
                             int32_t flags, void* stream);

/* Surrogate-ranked edge checks (no counterpart in the reference): as
 * csd_check_edges, but each edge's points are first scored by net `net` of
 * the surrogate bank `mlp` (csd_mlp_*, input dimension = the plant's); per
 * residue class k mod 32 the highest-scored point is a candidate, up to `top`
 * (<= 32) candidates are checked in decreasing score, then every other point
 * in the coarse-to-fine order of csd_check_edges. Verdicts are exact (a free
 * edge has every point checked); the ranking only moves a colliding edge's
 * first hit earlier. Points are scored in chunks of up to 2^22; an edge with
 * more points is checked unranked. starts/ends/free_out/points_checked follow
 * `flags`. */
typedef struct csd_mlp_s* csd_mlp_t;  /* the surrogate bank (csd_mlp_* below) */
csd_status_t csd_check_edges_ranked(csd_plant_t plant, csd_mlp_t mlp, int32_t net, const float* starts,
                                    const float* ends, int64_t n, float step_size, int32_t mode, int32_t top,
                                    uint8_t* free_out, int64_t* points_checked, int32_t flags, void* stream);

/* All-pairs visibility graph: VisibilityGraph, csdecomp/src/planning/cuda_visibility_graph.cu:175-375.
 * nodes: [n][dim] configurations (n >= 2). adjacency receives one byte per
 * pair i < j in upper-triangle row-major order (pair (i, j) at
 * i n - i (i + 1) / 2 + j - i - 1): 1 if the edge is collision free under the
 * reference's visibility-graph discretisation (CSD_EDGE_VG: both endpoints,
 * ceil(dist / step) + 2 points), else 0. Edges are generated on the device
 * from the node indices; each is checked by one warp with early exit. */
csd_status_t csd_visibility_graph(csd_plant_t plant, const float* nodes, int32_t n, float step_size,
                                  uint8_t* adjacency, int32_t flags, void* stream);

/* One pair: pairCollisionFree, csdecomp/src/plant/collision_checker.cpp:91-203
 * (GPU contact rule of cuda_geometry_utilities.h:16-125). 4x4 matrices column-major. */
csd_status_t csd_pair_collision_free(int32_t type_a, const float* dims_a, const float* X_L_B_a,
                                     const float* X_W_LA, int32_t type_b, const float* dims_b,
                                     const float* X_L_B_b, const float* X_W_LB, uint8_t* free_out);

/* Hit-and-run sampling in several polytopes: UniformSampleInHPolyhedronCuda,
 * csdecomp/src/geometry/cuda_hit_and_run_sampling.cu:137-210 (device-pointer
 * form executeUniformSampleInHPolyhedronKernel, :121-134). Polytope p owns rows
 * [face_offsets[p], face_offsets[p+1]) of A [F_total][dim] and b; starts:
 * [P][dim]; samples: [P][samples_per_polytope][dim]. Host-pointer calls check
 * every start point is contained (tolerance 1e-9, hpolyhedron.cpp:265-274).
 * A chain whose line search fails writes NaN (the reference leaves the slot
 * unwritten) and is counted in num_failed (optional, host int32). */
csd_status_t csd_uniform_sample_hpolyhedra(const float* A, const float* b, const int32_t* face_offsets,
                                           int32_t num_polytopes, int32_t dim, const float* starts,
                                           int32_t samples_per_polytope, int32_t mixing_steps, uint64_t seed,
                                           float* samples, int32_t* num_failed, int32_t flags, void* stream);

/* EizoOptions, csdecomp/src/planning/cuda_edge_inflation_zero_order.h:18-32. */
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
  int32_t verbose;
  int32_t track_iteration_information;
} csd_eizo_options_t;

/* EizoIterationInfo, cuda_edge_inflation_zero_order.h:37-47 (without the
 * plotting buffer). */
typedef struct {
  int32_t iteration_index;
  int32_t num_samples_drawn;
  int32_t collisions_threshold;
  int32_t num_collisions_unadaptive;
  int32_t num_collisions_updated;
  int32_t num_faces_placed;
  float iteration_time_ms;
} csd_eizo_iteration_info_t;

/* CudaEdgeInflator constructor, csdecomp/src/planning/cuda_polytope_builder.cu:70-109:
 * allocates all device memory once. domain: A [domain_faces][dim], b [domain_faces]
 * (host). face_capacity: maximum faces of a region (domain included). */
csd_status_t csd_inflator_create(csd_plant_t plant, const int32_t* robot_geometry_ids,
                                 int32_t num_robot_geometries, const csd_eizo_options_t* options,
                                 const float* domain_A, const float* domain_b, int32_t domain_faces,
                                 int32_t max_voxels, int32_t face_capacity, csd_inflator_t* out);
/* CudaEdgeInflator::inflateEdge, cuda_polytope_builder.cu:111-163, whose loop is
 * executeEizo, cuda_edge_inflation_zero_order.cu:94-339. Inputs are host arrays;
 * A_out/b_out (host) receive up to face_capacity rows; iteration records go to
 * info (host, may be NULL). */
csd_status_t csd_inflator_inflate(csd_inflator_t inflator, const float* line_start, const float* line_end,
                                  const float* voxels, int32_t num_voxels, float voxel_radius, float* A_out,
                                  float* b_out, int32_t* num_faces, csd_eizo_iteration_info_t* info,
                                  int32_t info_capacity, int32_t* num_iterations, void* stream);
/* EizoIterationInfo::points_post_bisection (cuda_edge_inflation_zero_order.h:46,
 * filled at :323-335 for dim <= 3): with track_iteration_information set and
 * dim <= 3, the collision points after bisection of iteration `iteration` of
 * the last csd_inflator_inflate ([count][dim], at most `capacity` rows
 * written); *count = 0 for an iteration without bisection or another dim. */
csd_status_t csd_inflator_points_post_bisection(csd_inflator_t inflator, int32_t iteration, float* points,
                                               int32_t capacity, int32_t* count);
csd_status_t csd_inflator_destroy(csd_inflator_t inflator);

/* EizoCuda one-shot form, cuda_edge_inflation_zero_order.cu:341-446: creates an
 * inflator, inflates, destroys it. */
csd_status_t csd_eizo(csd_plant_t plant, const float* line_start, const float* line_end, const float* voxels,
                      int32_t num_voxels, float voxel_radius, const float* domain_A, const float* domain_b,
                      int32_t domain_faces, const int32_t* robot_geometry_ids, int32_t num_robot_geometries,
                      const csd_eizo_options_t* options, int32_t face_capacity, float* A_out, float* b_out,
                      int32_t* num_faces, csd_eizo_iteration_info_t* info, int32_t info_capacity,
                      int32_t* num_iterations);

/* Batched EI-ZO (no counterpart in the reference, which inflates one edge per
 * executeEizo call, cuda_edge_inflation_zero_order.cu:94-339): up to max_slots
 * inflations, each with its own plant (one of `plants`, which must outlive the
 * batch), segment and domain, advance together through one persistent kernel
 * per stage, replayed as a CUDA graph. Each slot computes exactly what
 * csd_inflator_inflate computes for the same inputs. No voxels. */
typedef struct csd_batch_s* csd_batch_t;
/* csd_mlp_t (the surrogate bank, functions csd_mlp_* below) is declared above csd_check_edges_ranked. */
csd_status_t csd_batch_create(const csd_plant_t* plants, int32_t num_plants, int32_t max_slots,
                              const csd_eizo_options_t* options, int32_t face_capacity, csd_batch_t* out);
/* n inflations: inflation i uses plants[slot_plant[i]] (dim d_i);
 * starts/ends hold the segments back to back (d_i floats each); the domain of
 * inflation i is rows [domain_face_offsets[i], domain_face_offsets[i+1]) of
 * domain_b and the same rows of domain_A, stored back to back with d_i floats
 * per row. Region i is written to A_out at float offset sum_{j<i}
 * face_capacity * d_j (row-major, d_i floats per row) and b_out at i *
 * face_capacity; num_faces[i] rows. n may exceed max_slots: inflations
 * 0..max_slots-1 start at once and each later one starts in the first slot
 * that frees up (slots then run different iterations; each inflation still
 * computes exactly what csd_inflator_inflate computes). All arrays are host
 * memory; the call synchronises before returning. device_ms (optional)
 * receives the GPU time from the first to the last iteration. */
csd_status_t csd_batch_inflate(csd_batch_t batch, int32_t n, const int32_t* slot_plant, const float* starts,
                               const float* ends, const float* domain_A, const float* domain_b,
                               const int32_t* domain_face_offsets, float* A_out, float* b_out, int32_t* num_faces,
                               int32_t* num_iterations, float* device_ms);
/* Configurations the last csd_batch_inflate checked per slot (hit-and-run
 * samples plus bisection points), for throughput accounting. */
csd_status_t csd_batch_configs_checked(csd_batch_t h, int32_t n, int64_t* configs);

/* Profiling mode: while enabled, csd_batch_inflate launches each iteration's
 * stages one by one (no graph) with events between them and accumulates the
 * GPU time of each stage: [sample, score, sort, check, compact, bisect,
 * faces, step] (score and sort are zero without a surrogate). Enabling (or
 * disabling) resets the accumulators. */
csd_status_t csd_batch_set_profiling(csd_batch_t h, int32_t enable);
csd_status_t csd_batch_stage_ms(csd_batch_t h, float* stage_ms /* [8] */);
/* Autotuner: during the first `iterations` iterations of the next
 * csd_batch_inflate, every sampler variant (face pairs a lane holds at most x
 * resident blocks per SM: [8x1, 8x2, 8x3, 16x1, 16x2]) and every check
 * work-item cap ([8, 16, 32, 128, 512] configurations) is timed on that iteration's
 * own inputs; the fastest of each is kept for the graph and later calls. All
 * variants give identical samples. csd_batch_tuning reports the choice and
 * the summed time of each variant (variant_ms: 5 sampler entries, then 5 check
 * entries; *num_variants = 10). */
csd_status_t csd_batch_autotune(csd_batch_t h, int32_t iterations);
/* Surrogate-guided checking (mlp: one net per plant of the batch, same
 * dimensions; NULL turns it off). Each iteration then scores every sample
 * with the net, checks the samples in decreasing predicted collision
 * probability in rounds (csd_batch_set_surrogate_rounds), and stops checking a slot once its
 * admissibility is decided and, if inadmissible, num_particles collisions are
 * known or the next sample's predicted probability is below
 * stop_probability. Every verdict used is the exact checker's; the
 * admissibility test (first M samples) is unchanged; the bisected particles
 * are the first num_particles collisions found, in sample order (the plain
 * form's particles whenever no colliding sample was left unchecked). A slot
 * whose ordered check left fewer than 1/8 of its samples unchecked checks in
 * sample order (every sample, no scoring) for the rest of the call; once no
 * active slot orders, the call continues with the batched form's graph. */
csd_status_t csd_batch_set_surrogate(csd_batch_t h, csd_mlp_t mlp, float stop_probability);
/* Round schedule of the surrogate-guided check: round r covers sorted
 * positions up to first_round * (2^(r+1) - 1), the last round the rest
 * (defaults: 3 rounds, first round 1024 samples). */
csd_status_t csd_batch_set_surrogate_rounds(csd_batch_t h, int32_t rounds, int32_t first_round);
/* Sets the shapes directly (e.g. a tuning result kept from an earlier run):
 * sampler variant index as above, check work-item cap a multiple of 8. The
 * set variant then runs for every iteration. */
csd_status_t csd_batch_set_shapes(csd_batch_t h, int32_t sample_variant, int32_t check_item_cap);
/* Each sampler variant stages a slot's region (face-pair rows) in shared
 * memory up to a face count set by its blocks per SM (1: 5120 faces for dim
 * <= 8, 2844 above; 2: 2662 / 1478; 3: 1740 / 966); larger regions are read
 * from global memory through L1. After tuning, the first time an active slot
 * outgrows the running variant's staging, the next iteration times every
 * variant on its own inputs and the fastest runs from then on (kept for later
 * calls until csd_batch_autotune); when a region outgrows that variant's
 * staging too, the iterations continue with the fastest variant (by those
 * times) that stages the largest active region, else the roomiest (the graph
 * is captured once more per switch). tuned / large /
 * last_run: the tuned variant, the one the last switch chose for large
 * regions (before any switch: the one it would choose), the one the last
 * iteration ran. */
csd_status_t csd_batch_sample_variants(csd_batch_t h, int32_t* tuned, int32_t* large, int32_t* last_run);
/* Number of sampler variants and of check work-item caps the autotuner
 * chooses from (the index ranges of csd_batch_set_shapes and the entries of
 * csd_batch_tuning's variant_ms). Needs no device. No reference counterpart. */
void csd_batch_shape_counts(int32_t* num_sample_variants, int32_t* num_check_caps);
csd_status_t csd_batch_tuning(csd_batch_t h, int32_t* sample_variant, int32_t* check_item_cap, float* variant_ms,
                              int32_t* num_variants);
/* Profiling mode, last csd_batch_inflate: per iteration the eight stage times
 * (stage_ms[i * 8 + j]) and the slots active when it started; *count
 * receives the number of iterations (at most cap are written). */
csd_status_t csd_batch_iteration_profile(csd_batch_t h, int32_t cap, float* stage_ms, int32_t* active,
                                         int32_t* count);
/* Profiling mode, last csd_batch_inflate: per iteration the sampler variant
 * it ran (index as in csd_batch_set_shapes) and the most faces of a region
 * active when it started; *count receives the number of iterations. */
csd_status_t csd_batch_iteration_variants(csd_batch_t h, int32_t cap, int32_t* variant, int32_t* max_faces,
                                          int32_t* count);
/* Profiling mode, last csd_batch_inflate: algorithmic FLOPs of the sampling
 * stage, (2 d + 4) F per chain and mixing step (a . dir, the slack update and
 * the two theta-bound compares per face; FMA = 2, division not counted),
 * summed over the active slots' N_k chains of every iteration. */
csd_status_t csd_batch_sample_flops(csd_batch_t h, double* flops);
/* Kernels the last csd_batch_inflate launched (graph nodes counted per
 * replay, plus the autotuner's and the profiling mode's launches). No
 * reference counterpart. */
csd_status_t csd_batch_last_launches(csd_batch_t h, int64_t* launches);

csd_status_t csd_batch_destroy(csd_batch_t batch);

/* Allocation-free EI-ZO (no counterpart in the reference). Same inputs,
 * outputs and results as csd_eizo, for callers that must not allocate device
 * memory while they run (a real-time loop that owns a fixed memory budget, a
 * host that forbids allocation after start-up, code that has set aside all
 * device memory for itself): no cudaMalloc/cudaFree or other allocating call is
 * made. Its scratch is one 2 MiB array in the library's static device memory,
 * present on every device that loads the library until the process exits;
 * options whose scratch (samples of the unadaptive test, particles, region
 * faces, voxels, at most 2048 moving spheres and 1024 robot geometry ids)
 * exceeds it are rejected with CSD_ERR_CAPACITY. The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress); make that first
 * call before any stream capture. With CUDA's lazy module loading (the
 * default since CUDA 12.2) that first call, or the first kernel launch of the
 * library on a device, also loads the library's kernels and commits the
 * array: a caller that forbids allocation after start-up makes one call (a
 * warm-up inflation) per device during start-up. The cached address is tied
 * to the device's context: cudaDeviceReset after a call is not supported. All
 * calls share the one array, so calls that overlap on the GPU (several
 * streams or threads at once) race: issue them one at a time. The kernels
 * are csd_eizo's (the same sampler, checks, bisection and faces, so the same
 * regions bit for bit), except that voxels are tested one by one against
 * every robot geometry instead of through csd_eizo's per-call voxel hash
 * grid (2^18 configurations against 10,000 voxels on a B200: 85.4 ms instead
 * of 3.1 ms). Arrays are host memory; stream orders the work and is
 * synchronised before return. The plant is created beforehand with
 * csd_plant_create. */
csd_status_t csd_eizo_noalloc(csd_plant_t plant, const float* line_start, const float* line_end,
                              const float* voxels, int32_t num_voxels, float voxel_radius, const float* domain_A,
                              const float* domain_b, int32_t domain_faces, const int32_t* robot_geometry_ids,
                              int32_t num_robot_geometries, const csd_eizo_options_t* options, int32_t face_capacity,
                              float* A_out, float* b_out, int32_t* num_faces, csd_eizo_iteration_info_t* info,
                              int32_t info_capacity, int32_t* num_iterations, void* stream);

/* EditRegionsOptions, csdecomp/src/planning/cuda_edit_regions.h:12-16
 * (defaults 0.01, 9; verbose printing is left to the caller). */
typedef struct {
  float configuration_margin;
  uint32_t bisection_steps;
} csd_edit_regions_options_t;

/* Region editing: EditRegionsCuda, csdecomp/src/planning/cuda_edit_regions.cu:44-301
 * (pybind cuda_bindings.h:140-179). Collision i ([n][dim]) belongs to segment
 * line_segment_idxs[i] < m; segment r runs from line_starts[r] to
 * line_ends[r] ([m][dim]) and lies in region r, rows
 * [face_offsets[r], face_offsets[r+1]) of A ([F][dim] row-major) and b. Each
 * collision is bisected towards its projection on its segment
 * (bisection_steps fused FK + checks, voxels as in csd_check_points); per
 * region a face is placed for each optimized collision, nearest first, that
 * lies strictly inside the region edited so far, relaxed so the segment stays
 * inside. A_out/b_out hold face_offsets[m] + n rows: region r is written at
 * row face_offsets[r] + (collisions of segments < r), num_faces[r] rows (the
 * original faces first); other rows are unspecified. projections and
 * optimized_collisions ([n][dim]) come back grouped by segment, in the given
 * order within a segment, as the reference returns them. Errors: endpoints
 * outside their region (CSD_ERR_NOT_CONTAINED), n = 0, a segment index out of
 * range, no robot geometry ids or voxel_radius <= 0 (CSD_ERR_INVALID), more
 * than 10000 voxels (CSD_ERR_CAPACITY). Host arrays; synchronous. */
csd_status_t csd_edit_regions(csd_plant_t plant, const float* collisions, const uint32_t* line_segment_idxs,
                              int64_t n, const float* line_starts, const float* line_ends, int32_t m,
                              const float* A, const float* b, const int32_t* face_offsets, const float* voxels,
                              int32_t num_voxels, float voxel_radius, const int32_t* robot_geometry_ids,
                              int32_t num_robot_geometries, const csd_edit_regions_options_t* options,
                              float* A_out, float* b_out, int32_t* num_faces, float* projections,
                              float* optimized_collisions);

/* numSamplesUnadaptive, csdecomp/src/planning/cuda_set_builder_utils.h:198-203. */
uint32_t csd_num_samples_unadaptive(float epsilon, float delta, float tau);

/* Diagnostics (no counterpart in the reference): FP32 FMA throughput of the
 * current device, the denominator of the collision kernels' roofline. */
csd_status_t csd_fp32_fma_probe(int64_t iters, double* flops, double* seconds);
/* Link-level broad phase of the collision checks (no counterpart in the
 * reference, which tests every pair): per configuration, each moving link's
 * bounding sphere is placed in the world and pairs whose link or static
 * bounding spheres are apart by more than 1e-4 m are skipped. Verdicts are
 * unchanged. On by default for plants with at most 32 moving links and 1024
 * static geometries; enable = 0 evaluates every pair (the full sweep that
 * csd_plant_flops counts). Takes effect for later calls and for batches
 * created afterwards. */
csd_status_t csd_plant_set_culling(csd_plant_t plant, int32_t enable);
/* Voxel hash grid of the voxel checks (csd_check_points with voxels, csd_eizo
 * and csd_inflator_inflate with voxels, csd_edit_regions; the reference tests
 * every robot geometry against every voxel, cuda_collision_checker.cu:374-435):
 * per call the voxels are bucketed on the device by a spatial hash of their
 * cells, and each robot geometry tests only the voxels in the cells its
 * bounding sphere touches. Used for 64 voxels or more; verdicts are
 * unchanged. On by default; enable = 0 tests every voxel. */
csd_status_t csd_plant_set_voxel_grid(csd_plant_t plant, int32_t enable);

/* Algorithmic FP32 work of checking one configuration of this plant without
 * early exit: forward kinematics, geometry placement and all pair tests
 * (FMA = 2 FLOP; sqrt, division and sincos not counted). */
csd_status_t csd_plant_flops(csd_plant_t plant, double* fk_flops, double* placement_flops, double* pair_flops);

/* ------------------------------------------------------------------------
 * Collision-likelihood surrogate (no counterpart in the reference): a bank of
 * BF16 MLPs, in -> 256 -> 256 -> 256 -> 1 with ReLU and FP32 accumulation, one
 * per plant, run by hand-written tcgen05 kernels. Inputs are scaled by
 * in_scale (1/pi maps [-pi, pi] joint limits to [-1, 1]) and zero padded to
 * 16. Parameters per net (csd_mlp_num_params floats): W1 [256][16], b1 [256],
 * W2 [256][256], b2, W3 [256][256], b3, w4 [256], b4 [1] (row-major
 * [out][in]). The logit is P(collision) before the sigmoid.
 * ------------------------------------------------------------------------ */
int32_t csd_mlp_num_params(void);
csd_status_t csd_mlp_create(int32_t nets, const int32_t* dims, float in_scale, uint64_t seed, csd_mlp_t* out);
csd_status_t csd_mlp_destroy(csd_mlp_t mlp);
csd_status_t csd_mlp_get_params(csd_mlp_t mlp, float* params /* [nets][num_params] */);
csd_status_t csd_mlp_set_params(csd_mlp_t mlp, const float* params);
/* Logits of `groups` row blocks: block i has rows[i] rows of dims[net[i]]
 * floats in x (blocks concatenated); logits likewise. flags: CSD_PTR_*. */
csd_status_t csd_mlp_infer(csd_mlp_t mlp, int32_t groups, const int32_t* net, const int32_t* rows, const float* x,
                           float* logits, int32_t flags, void* stream);
/* One forward + backward pass (mean binary cross-entropy with logits) on a
 * host batch of `batch` rows per net (x [nets][batch][dim], y [nets][batch]
 * 0/1); gradients [nets][num_params] and per-net loss to host. batch is a
 * multiple of 32. */
csd_status_t csd_mlp_gradients(csd_mlp_t mlp, const float* x, const uint8_t* y, int32_t batch, float* grads,
                               float* loss);
/* Adam training, `steps` minibatches of `batch` rows per net taken in order
 * from device arrays x [nets][n][dim] and y [nets][n] (n a multiple of batch;
 * shuffle beforehand); loss_history (host, optional) receives the mean loss of
 * every step. */
csd_status_t csd_mlp_train(csd_mlp_t mlp, const float* x, const uint8_t* y, int32_t n, int32_t batch, int32_t steps,
                           float lr, float* loss_history, void* stream);
/* Test hook: D [M][N] f32 = A [M][K] * B [N][K]^T for bf16 bit patterns
 * (N = 16 or 256, K a multiple of 8) through the tensor-core GEMM. */
csd_status_t csd_mlp_gemm_test(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, float* D);

#ifdef __cplusplus
}
#endif
#endif
