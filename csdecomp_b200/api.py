"""Python API with the reference's names (csdecomp/src/pybind/csdecomp/*.h).

Array conventions follow the pybind bindings: a batch of configurations is
a ``dim x N`` matrix (one configuration per column), voxels are ``3 x V``,
polytopes are ``A`` (faces x dim) and ``b``. Every function runs on the GPU
through libcsdecomp_b200.so; host arrays are copied in and out by the
library, device-resident work goes through ``csdecomp_b200.device``.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _capi as C
from .plant import (CollisionGeometry, MinimalKinematicTree, MinimalPlant)

MAX_NUM_FACES = 4000      # hpolyhedron.h:5 (default face capacity of a region)
MAX_DIM = 16              # this build's limit (the reference's MAX_DIM is 14)
MAX_NUM_VOXELS = 10000    # cuda_edge_inflation_zero_order.h:13


# --------------------------------------------------------------------- plant handles
def plant_handle(plant: MinimalPlant) -> C.PlantHandle:
    """Device tables of a plant, created on first use and cached on the plant."""
    h = getattr(plant, "_csd_handle", None)
    if h is None or getattr(plant, "_csd_handle_pairs", None) is not plant._pairs:
        kt = plant.kin_tree
        h = C.PlantHandle(plant.arrays(), kt.num_joints, kt.num_links, kt.num_configuration_variables,
                          plant.num_scene_geometries, plant.num_collision_pairs)
        plant._csd_handle = h
        plant._csd_handle_pairs = plant._pairs
    return h


def _tree_plant(tree: MinimalKinematicTree) -> MinimalPlant:
    return MinimalPlant(tree, [], np.zeros((2, 0), np.int32))


def _configs(configurations: np.ndarray, dim: int) -> np.ndarray:
    """dim x N (reference layout) -> contiguous [N][dim] float32."""
    q = np.asarray(configurations, dtype=np.float32)
    if q.ndim == 1:
        q = q.reshape(dim, 1)
    if q.shape[0] != dim:
        raise RuntimeError(f"incorrect number of configuration variables: expected {dim}, got {q.shape[0]}")
    return np.ascontiguousarray(q.T)


class Voxels:
    """VoxelsWrapper (pybind/csdecomp/voxel_wrapper.h): a 3 x V matrix of voxel centres."""

    def __init__(self, matrix: Optional[np.ndarray] = None):
        self.matrix = np.zeros((3, 0), np.float32) if matrix is None else np.asarray(matrix, np.float32).reshape(3, -1)

    def set_matrix(self, m: np.ndarray) -> None:
        self.matrix = np.asarray(m, np.float32).reshape(3, -1)

    def get_matrix(self) -> np.ndarray:
        return self.matrix


def _voxel_rows(voxels) -> np.ndarray:
    m = voxels.matrix if isinstance(voxels, Voxels) else (np.zeros((3, 0)) if voxels is None else voxels)
    m = np.asarray(m, np.float32).reshape(3, -1)
    return np.ascontiguousarray(m.T)


# ------------------------------------------------------------------ collision checks
def CheckCollisionFreeCuda(configurations: np.ndarray, plant: MinimalPlant) -> np.ndarray:
    """checkCollisionFreeCuda (cuda_collision_checker.cu:437-487): uint8 per
    configuration, 1 = collision free."""
    h = plant_handle(plant)
    q = _configs(configurations, h.dim)
    out = np.zeros(q.shape[0], np.uint8)
    C.check(C.lib().csd_check_points(h.handle, C.ptr(q), ctypes.c_int64(q.shape[0]), None, 0, ctypes.c_float(0),
                                     None, 0, C.ptr(out), C.CSD_PTR_HOST, None))
    return out


def CheckCollisionFreeVoxelsCuda(configurations: np.ndarray, voxels, voxel_radius: float, plant: MinimalPlant,
                                 robot_geometries: Sequence[int]) -> np.ndarray:
    """checkCollisionFreeVoxelsCuda (cuda_collision_checker.cu:374-435)."""
    h = plant_handle(plant)
    q = _configs(configurations, h.dim)
    v = _voxel_rows(voxels)
    ids = np.ascontiguousarray(np.asarray(list(robot_geometries), np.int32).reshape(-1))
    out = np.zeros(q.shape[0], np.uint8)
    C.check(C.lib().csd_check_points(h.handle, C.ptr(q), ctypes.c_int64(q.shape[0]), C.ptr(v), v.shape[0],
                                     ctypes.c_float(voxel_radius), C.ptr(ids), ids.size, C.ptr(out),
                                     C.CSD_PTR_HOST, None))
    return out


def CheckCollisionFree(configuration: np.ndarray, plant: MinimalPlant) -> bool:
    """checkCollisionFree (collision_checker.cpp:9-39), evaluated on the GPU."""
    return bool(CheckCollisionFreeCuda(np.asarray(configuration, np.float32).reshape(-1, 1), plant)[0])


def CheckCollisionFreeVoxels(configuration: np.ndarray, voxels, voxel_radius: float, plant: MinimalPlant,
                             robot_geometry_index: Sequence[int]) -> bool:
    """checkCollisionFreeVoxels (collision_checker.cpp:55-89), evaluated on the GPU."""
    for g in robot_geometry_index:
        if g >= plant.num_scene_geometries:
            raise RuntimeError("Invalid robot geometry ID, check the SceneInspector for vaild ids.")
    return bool(CheckCollisionFreeVoxelsCuda(np.asarray(configuration, np.float32).reshape(-1, 1), voxels,
                                             voxel_radius, plant, robot_geometry_index)[0])


def CheckEdgesCollisionFreeCuda(starts: np.ndarray, ends: np.ndarray, plant: MinimalPlant, step_size: float = 0.01,
                                discretization: int = C.CSD_EDGE_L2_REF, return_points_checked: bool = False):
    """Batched edge check with early exit. starts/ends are dim x E. The default
    discretisation is checkEdgeCollisionFree's (collision_checker.cpp:41-53)."""
    h = plant_handle(plant)
    s = _configs(starts, h.dim)
    e = _configs(ends, h.dim)
    if s.shape != e.shape:
        raise RuntimeError("starts and ends must have the same shape")
    out = np.zeros(s.shape[0], np.uint8)
    pts = np.zeros(s.shape[0], np.int64) if return_points_checked else None
    C.check(C.lib().csd_check_edges(h.handle, C.ptr(s), C.ptr(e), ctypes.c_int64(s.shape[0]),
                                    ctypes.c_float(step_size), discretization, C.ptr(out), C.ptr(pts),
                                    C.CSD_PTR_HOST, None))
    return (out, pts) if return_points_checked else out


def CheckEdgesCollisionFreeRankedCuda(starts: np.ndarray, ends: np.ndarray, plant: MinimalPlant, surrogate, net: int = 0,
                                      step_size: float = 0.01, discretization: int = C.CSD_EDGE_L2_REF, top: int = 8,
                                      return_points_checked: bool = False):
    """CheckEdgesCollisionFreeCuda with each edge's points ordered by a
    CollisionSurrogate (net `net`): the `top` highest-scored candidates are
    checked first, then the rest coarse-to-fine. Verdicts are exact and equal
    CheckEdgesCollisionFreeCuda's; colliding edges usually exit after fewer
    points (csd_check_edges_ranked)."""
    h = plant_handle(plant)
    s = _configs(starts, h.dim)
    e = _configs(ends, h.dim)
    if s.shape != e.shape:
        raise RuntimeError("starts and ends must have the same shape")
    out = np.zeros(s.shape[0], np.uint8)
    pts = np.zeros(s.shape[0], np.int64) if return_points_checked else None
    C.check(C.lib().csd_check_edges_ranked(h.handle, surrogate.handle, int(net), C.ptr(s), C.ptr(e),
                                           ctypes.c_int64(s.shape[0]), ctypes.c_float(step_size), discretization,
                                           int(top), C.ptr(out), C.ptr(pts), C.CSD_PTR_HOST, None))
    return (out, pts) if return_points_checked else out


def CheckEdgeCollisionFree(configuration_1: np.ndarray, configuration_2: np.ndarray, plant: MinimalPlant,
                           step_size: float = 0.01) -> bool:
    """checkEdgeCollisionFree (collision_checker.cpp:41-53), evaluated on the GPU."""
    return bool(CheckEdgesCollisionFreeCuda(np.asarray(configuration_1, np.float32).reshape(-1, 1),
                                            np.asarray(configuration_2, np.float32).reshape(-1, 1), plant,
                                            step_size)[0])


def VisibilityGraph(configurations: np.ndarray, plant: MinimalPlant, step_size: float,
                    max_configs_per_batch: int = 10000000):
    """VisibilityGraph (cuda_visibility_graph.cu:175-375): the collision-free
    edges among the columns of `configurations` (dim x n) as an n x n
    scipy.sparse matrix with a 1 at (i, j), i < j, for every free edge (the
    upper triangle, as the reference's triplets). Edges use the reference's
    visibility-graph discretisation (both endpoints, ceil(dist/step) + 2
    points). The edges are generated and checked on the device, so
    max_configs_per_batch (the reference's batching knob) only has its range
    checked."""
    import scipy.sparse as sp
    h = plant_handle(plant)
    q = _configs(configurations, h.dim)
    n = q.shape[0]
    if n < 2:
        raise ValueError("a visibility graph needs at least two configurations")
    if not step_size >= 1e-12:
        raise ValueError("step_size must be at least 1e-12")
    if not 1 < max_configs_per_batch <= 10000000:
        raise ValueError("max_configs_per_batch must be in (1, 1e7]")
    E = n * (n - 1) // 2
    adj = np.zeros(E, np.uint8)
    C.check(C.lib().csd_visibility_graph(h.handle, C.ptr(q), n, ctypes.c_float(step_size), C.ptr(adj),
                                         C.CSD_PTR_HOST, None))
    iu, ju = np.triu_indices(n, 1)
    keep = adj.astype(bool)
    return sp.csr_matrix((np.ones(int(keep.sum()), np.uint8), (iu[keep], ju[keep])), shape=(n, n))


def PairCollisionFree(geom_a: CollisionGeometry, x_w_la: np.ndarray, geom_b: CollisionGeometry,
                      x_w_lb: np.ndarray) -> bool:
    """pairCollisionFree (collision_checker.cpp:91-203)."""
    def cm(x):
        return np.ascontiguousarray(np.asarray(x, np.float32).reshape(4, 4).T.reshape(-1))
    out = np.zeros(1, np.uint8)
    da = np.ascontiguousarray(geom_a.dimensions, np.float32)
    db = np.ascontiguousarray(geom_b.dimensions, np.float32)
    C.check(C.lib().csd_pair_collision_free(int(geom_a.type), C.ptr(da), C.ptr(cm(geom_a.X_L_B)), C.ptr(cm(x_w_la)),
                                            int(geom_b.type), C.ptr(db), C.ptr(cm(geom_b.X_L_B)), C.ptr(cm(x_w_lb)),
                                            C.ptr(out)))
    return bool(out[0])


def ComputeForwardKinematicsCuda(configurations: np.ndarray, plant) -> np.ndarray:
    """computeForwardKinematicsCuda (cuda_forward_kinematics.cu:92-129):
    returns [N][num_links][4][4] link-to-world transforms."""
    if isinstance(plant, MinimalKinematicTree):
        plant = _tree_plant(plant)
    h = plant_handle(plant)
    q = _configs(configurations, h.dim)
    out = np.zeros((q.shape[0], h.num_links, 16), np.float32)
    C.check(C.lib().csd_fk(h.handle, C.ptr(q), ctypes.c_int64(q.shape[0]), C.ptr(out), C.CSD_PTR_HOST, None))
    return np.ascontiguousarray(out.reshape(q.shape[0], h.num_links, 4, 4).transpose(0, 1, 3, 2))


def computeLinkFrameToWorldTransformsMinimal(joint_values: np.ndarray, tree: MinimalKinematicTree) -> np.ndarray:
    """Binding of computeLinkFrameToWorldTransformsMinimal (plant_bindings.h:174-185):
    a (4 * num_links) x 4 matrix of stacked link-to-world transforms."""
    tf = ComputeForwardKinematicsCuda(np.asarray(joint_values, np.float32).reshape(-1, 1), tree)[0]
    return tf.reshape(-1, 4)


# --------------------------------------------------------------------- polytopes
class MinimalHPolyhedron:
    """MinimalHPolyhedron (hpolyhedron.h:15-21): A row-major, b, num_faces, dim."""

    def __init__(self, A: Optional[np.ndarray] = None, b: Optional[np.ndarray] = None):
        self._A = np.zeros((0, 0), np.float32) if A is None else np.asarray(A, np.float32)
        self._b = np.zeros(0, np.float32) if b is None else np.asarray(b, np.float32).reshape(-1)

    def A(self) -> np.ndarray:
        return self._A.copy()

    def b(self) -> np.ndarray:
        return self._b.copy()

    @property
    def num_faces(self) -> int:
        return int(self._A.shape[0])

    @property
    def dim(self) -> int:
        return int(self._A.shape[1]) if self._A.ndim == 2 else 0


class HPolyhedron:
    """{x : A x <= b} (hpolyhedron.h:48-118)."""

    _sample_calls = 0

    def __init__(self, A=None, b=None):
        if isinstance(A, MinimalHPolyhedron):
            self._A, self._b = A.A(), A.b()
        elif A is None:
            self._A, self._b = np.zeros((0, 0), np.float32), np.zeros(0, np.float32)
        else:
            A = np.asarray(A, np.float32)
            b = np.asarray(b, np.float32).reshape(-1)
            if A.shape[0] != b.shape[0]:
                raise ValueError("A and b dimensions do not match")
            self._A, self._b = A.copy(), b.copy()

    def A(self) -> np.ndarray:
        return self._A

    def b(self) -> np.ndarray:
        return self._b

    def ambient_dimension(self) -> int:
        return int(self._A.shape[1]) if self._A.ndim == 2 else 0

    def MakeBox(self, lower_limit, upper_limit) -> None:
        """hpolyhedron.cpp:104-122: faces (-e_i, -lo_i), (e_i, hi_i) interleaved."""
        lo = np.asarray(lower_limit, np.float32).reshape(-1)
        hi = np.asarray(upper_limit, np.float32).reshape(-1)
        if lo.size != hi.size:
            raise ValueError("Lower and upper limits must have the same dimension")
        d = lo.size
        A = np.zeros((2 * d, d), np.float32)
        b = np.zeros(2 * d, np.float32)
        for i in range(d):
            A[2 * i, i], A[2 * i + 1, i] = -1, 1
            b[2 * i], b[2 * i + 1] = -lo[i], hi[i]
        self._A, self._b = A, b

    def GetMyMinimalHPolyhedron(self) -> MinimalHPolyhedron:
        return MinimalHPolyhedron(self._A, self._b)

    def PointInSet(self, point, tol: float = 1e-9) -> bool:
        """hpolyhedron.cpp:265-274 (FP32 arithmetic)."""
        x = np.asarray(point, np.float32).reshape(-1)
        if x.size != self.ambient_dimension():
            raise ValueError("Point dimension does not match polyhedron dimension")
        return bool(np.all(self._A @ x <= self._b + np.float32(tol)))

    def UniformSample(self, previous_sample, mixing_steps: int) -> np.ndarray:
        """Hit-and-run from previous_sample (hpolyhedron.cpp:179-230), on the GPU;
        each call draws a fresh stream."""
        HPolyhedron._sample_calls += 1
        s = UniformSampleInHPolyhedraCuda([self], np.asarray(previous_sample, np.float32).reshape(-1, 1), 1,
                                          mixing_steps, seed=1337 + HPolyhedron._sample_calls)
        return s[0][:, 0]

    def ChebyshevCenter(self) -> np.ndarray:
        """Centre of the largest inscribed ball (hpolyhedron.cpp:124-155), by LP."""
        from scipy.optimize import linprog
        A = self._A.astype(np.float64)
        n = A.shape[1]
        Ac = np.hstack([A, np.linalg.norm(A, axis=1, keepdims=True)])
        c = np.zeros(n + 1)
        c[-1] = -1
        res = linprog(c, A_ub=Ac, b_ub=self._b.astype(np.float64), bounds=[(None, None)] * n + [(0, None)])
        if not res.success:
            raise RuntimeError("Failed to solve LP for Chebyshev center")
        return res.x[:n].astype(np.float32)

    def GetFeasiblePoint(self) -> np.ndarray:
        return self.ChebyshevCenter()


def UniformSampleInHPolyhedraCuda(polyhedra: Sequence[HPolyhedron], starting_points: np.ndarray,
                                  num_samples_per_hpolyhedron: int, mixing_steps: int, seed: int = 1337):
    """UniformSampleInHPolyhedronCuda (cuda_hit_and_run_sampling.cu:137-210):
    a list of dim x S sample matrices, one per polytope."""
    polys = list(polyhedra)
    if not polys:
        return []
    dim = polys[0].ambient_dimension()
    sp = np.asarray(starting_points, np.float32)
    if sp.ndim == 1:
        sp = sp.reshape(-1, 1)
    if sp.shape[0] != dim:
        raise RuntimeError("starting points have wrong dimension!")
    if sp.shape[1] != len(polys):
        raise RuntimeError(f"Incorrect number of starting points supplied. A total of {len(polys)} polyhedra "
                           f"and {sp.shape[1]} starting points were passed to the sampler. ")
    A = np.ascontiguousarray(np.concatenate([p.A().reshape(-1, dim) for p in polys]), np.float32)
    b = np.ascontiguousarray(np.concatenate([p.b() for p in polys]), np.float32)
    off = np.zeros(len(polys) + 1, np.int32)
    off[1:] = np.cumsum([p.A().shape[0] for p in polys])
    starts = np.ascontiguousarray(sp.T)
    S = int(num_samples_per_hpolyhedron)
    out = np.zeros((len(polys), S, dim), np.float32)
    nf = ctypes.c_int32(0)
    C.check(C.lib().csd_uniform_sample_hpolyhedra(C.ptr(A), C.ptr(b), C.ptr(off), len(polys), dim, C.ptr(starts), S,
                                                  int(mixing_steps), ctypes.c_uint64(seed & (2 ** 64 - 1)),
                                                  C.ptr(out), ctypes.byref(nf), C.CSD_PTR_HOST, None))
    return [np.ascontiguousarray(out[i].T) for i in range(len(polys))]


# -------------------------------------------------------------------------- EI-ZO
@dataclass
class EizoOptions:
    """EizoOptions (cuda_edge_inflation_zero_order.h:18-32), same fields and defaults."""
    configuration_margin: float = 0.01
    tau: float = 0.5
    delta: float = 0.05
    epsilon: float = 0.01
    bisection_steps: int = 9
    num_particles: int = 1000
    max_hyperplanes_per_iteration: int = 10
    max_iterations: int = 500
    mixing_steps: int = 40
    seed: int = 1337
    verbose: bool = False
    track_iteration_information: bool = True

    def _c(self) -> C.EizoOptionsC:
        return C.EizoOptionsC(self.configuration_margin, self.tau, self.delta, self.epsilon, self.bisection_steps,
                              self.num_particles, self.max_hyperplanes_per_iteration, self.max_iterations,
                              self.mixing_steps, self.seed, int(self.verbose), int(self.track_iteration_information))


@dataclass
class EizoIterationInfo:
    iteration_index: int = 0
    num_samples_drawn: int = 0
    collisions_threshold: int = 0
    num_collisions_unadaptive: int = 0
    num_collisions_updated: int = 0
    num_faces_placed: int = 0
    iteration_time_ms: float = 0.0
    # dim x K collision points after bisection (cuda_edge_inflation_zero_order.h:46); kept, as the
    # reference keeps them, only with track_iteration_information and dim <= 3, else empty
    points_post_bisection: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), np.float32))


@dataclass
class EizoInfo:
    iteration_info: List[EizoIterationInfo] = field(default_factory=list)


def printEizoSummary(info: EizoInfo) -> None:
    """printEizoSummary (cuda_edge_inflation_zero_order.h:168-213)."""
    print("EI-ZO Summary:\n=============================")
    print(f"Total iterations: {len(info.iteration_info)}\n")
    print(f"{'Iter.':<8}{'Samples':<10}{'Col. (UT)':<12}{'Thresh.':<10}{'Col. (OPT)':<12}{'Faces':<8}{'Time (ms)':<12}")
    print("-" * 72)
    for it in info.iteration_info:
        print(f"{it.iteration_index:<8}{it.num_samples_drawn:<10}{it.num_collisions_unadaptive:<12}"
              f"{it.collisions_threshold:<10}{it.num_collisions_updated:<12}{it.num_faces_placed:<8}"
              f"{it.iteration_time_ms:<12.2f}")
    print("-" * 72)


def numSamplesUnadaptive(epsilon: float, delta: float, tau: float) -> int:
    """cuda_set_builder_utils.h:198-203."""
    return int(C.lib().csd_num_samples_unadaptive(epsilon, delta, tau))


class CudaEdgeInflator:
    """CudaEdgeInflator (cuda_polytope_builder.h:16-44): allocates once, then
    inflateEdge reuses the device memory."""

    def __init__(self, plant: MinimalPlant, robot_geometry_ids: Sequence[int], options: EizoOptions,
                 domain: HPolyhedron, face_capacity: int = MAX_NUM_FACES, max_voxels: int = MAX_NUM_VOXELS):
        self._plant = plant
        self._h = plant_handle(plant)
        if domain.ambient_dimension() != self._h.dim:
            raise RuntimeError("domain dimension does not match the plant")
        self._domain = domain
        self._options = options
        self._capacity = int(face_capacity)
        ids = np.ascontiguousarray(np.asarray(list(robot_geometry_ids), np.int32).reshape(-1))
        A = np.ascontiguousarray(domain.A(), np.float32)
        b = np.ascontiguousarray(domain.b(), np.float32)
        self._opt_c = options._c()
        h = ctypes.c_void_p()
        C.check(C.lib().csd_inflator_create(self._h.handle, C.ptr(ids), ids.size, ctypes.byref(self._opt_c),
                                            C.ptr(A), C.ptr(b), A.shape[0], int(max_voxels), self._capacity,
                                            ctypes.byref(h)))
        self._handle = h
        self._A_out = np.zeros((self._capacity, self._h.dim), np.float32)
        self._b_out = np.zeros(self._capacity, np.float32)
        self._iters = (C.EizoIterC * max(1, int(options.max_iterations)))()
        self.last_info = EizoInfo()

    def inflateEdge(self, line_start, line_end, voxels=None, voxel_radius: float = 0.0,
                    verbose: bool = True) -> HPolyhedron:
        d = self._h.dim
        ls = np.ascontiguousarray(np.asarray(line_start, np.float32).reshape(-1))
        le = np.ascontiguousarray(np.asarray(line_end, np.float32).reshape(-1))
        if ls.size != d or le.size != d:
            raise RuntimeError("line segment has the wrong dimension")
        v = _voxel_rows(voxels)
        nf = ctypes.c_int32(0)
        nit = ctypes.c_int32(0)
        C.check(C.lib().csd_inflator_inflate(self._handle, C.ptr(ls), C.ptr(le), C.ptr(v) if v.size else None,
                                             v.shape[0], ctypes.c_float(voxel_radius), C.ptr(self._A_out),
                                             C.ptr(self._b_out), ctypes.byref(nf), self._iters,
                                             len(self._iters), ctypes.byref(nit), None))
        info = EizoInfo([EizoIterationInfo(*[getattr(self._iters[i], n) for n, _ in C.EizoIterC._fields_])
                         for i in range(nit.value)])
        if d <= 3 and self._options.track_iteration_information:
            for i, it in enumerate(info.iteration_info):
                cnt = ctypes.c_int32(0)
                C.check(C.lib().csd_inflator_points_post_bisection(self._handle, i, None, 0, ctypes.byref(cnt)))
                if cnt.value:
                    pts = np.zeros((cnt.value, d), np.float32)
                    C.check(C.lib().csd_inflator_points_post_bisection(self._handle, i, C.ptr(pts), cnt.value,
                                                                       ctypes.byref(cnt)))
                    it.points_post_bisection = np.ascontiguousarray(pts.T)
        self.last_info = info
        if verbose:
            print("======================== Set builder ===========================")
            printEizoSummary(info)
            print("===================== End Set builder ===========================")
        return HPolyhedron(self._A_out[:nf.value].copy(), self._b_out[:nf.value].copy())

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h and C._lib is not None:
            try:
                C._lib.csd_inflator_destroy(h)
            except Exception:  # pragma: no cover
                pass
        self._handle = None


def EizoCuda(line_start, line_end, voxels, voxel_radius: float, domain: HPolyhedron, plant: MinimalPlant,
             robot_geometry_ids: Sequence[int], options: EizoOptions,
             eizo_info: Optional[EizoInfo] = None, face_capacity: int = MAX_NUM_FACES) -> MinimalHPolyhedron:
    """EizoCuda one-shot form (cuda_edge_inflation_zero_order.cu:341-446)."""
    h = plant_handle(plant)
    d = h.dim
    ls = np.ascontiguousarray(np.asarray(line_start, np.float32).reshape(-1))
    le = np.ascontiguousarray(np.asarray(line_end, np.float32).reshape(-1))
    v = _voxel_rows(voxels)
    ids = np.ascontiguousarray(np.asarray(list(robot_geometry_ids), np.int32).reshape(-1))
    A = np.ascontiguousarray(domain.A(), np.float32)
    b = np.ascontiguousarray(domain.b(), np.float32)
    A_out = np.zeros((face_capacity, d), np.float32)
    b_out = np.zeros(face_capacity, np.float32)
    iters = (C.EizoIterC * max(1, int(options.max_iterations)))()
    nf, nit = ctypes.c_int32(0), ctypes.c_int32(0)
    o = options._c()
    C.check(C.lib().csd_eizo(h.handle, C.ptr(ls), C.ptr(le), C.ptr(v) if v.size else None, v.shape[0],
                             ctypes.c_float(voxel_radius), C.ptr(A), C.ptr(b), A.shape[0], C.ptr(ids), ids.size,
                             ctypes.byref(o), face_capacity, C.ptr(A_out), C.ptr(b_out), ctypes.byref(nf), iters,
                             len(iters), ctypes.byref(nit)))
    if eizo_info is not None:
        eizo_info.iteration_info = [EizoIterationInfo(*[getattr(iters[i], n) for n, _ in C.EizoIterC._fields_])
                                    for i in range(nit.value)]
    return MinimalHPolyhedron(A_out[:nf.value].copy(), b_out[:nf.value].copy())


class EditRegionsOptions:
    """EditRegionsOptions (cuda_edit_regions.h:12-16)."""

    def __init__(self, configuration_margin: float = 0.01, bisection_steps: int = 9, verbose: bool = False):
        self.configuration_margin = configuration_margin
        self.bisection_steps = bisection_steps
        self.verbose = verbose

    def _c(self) -> "C.EditRegionsOptionsC":
        if int(self.bisection_steps) < 0:
            raise ValueError("bisection_steps must be non-negative")
        return C.EditRegionsOptionsC(float(self.configuration_margin), int(self.bisection_steps))


def EditRegionsCuda(collisions, line_segment_idxs, line_start_points, line_end_points, regions, plant,
                    robot_geometry_ids, voxels, voxel_radius: float, options: EditRegionsOptions):
    """EditRegionsCuda (cuda_edit_regions.cu:44-301, binding cuda_bindings.h:140-179):
    cuts the colliding configurations (columns of `collisions`, dim x n) out of
    the regions while each region keeps its segment (columns of
    line_start_points / line_end_points, dim x len(regions)). Collision i is
    bisected towards its projection on segment line_segment_idxs[i]; faces are
    placed nearest first, each only if its optimized collision is still inside
    the region. Returns (edited regions, (projections, optimized collisions)),
    the two dim x n matrices grouped by segment as the reference returns them."""
    h = plant_handle(plant)
    d = h.dim
    regions = list(regions)
    if not regions:
        raise ValueError("Regions vector cannot be empty")
    m = len(regions)
    ls = np.asarray(line_start_points, np.float32)
    le = np.asarray(line_end_points, np.float32)
    if ls.ndim != 2 or le.ndim != 2 or ls.shape[1] != m or le.shape[1] != m:
        raise ValueError("Number of line segments must match number of regions")
    if ls.shape[0] != le.shape[0]:
        raise ValueError("Line start and end points must have same dimension")
    amb = regions[0].ambient_dimension()
    col = np.asarray(collisions, np.float32)
    if col.ndim != 2 or col.shape[0] != amb:
        raise ValueError("collisions must live in the same space as the regions")
    if ls.shape[0] != amb:
        raise ValueError("the linesegments must live in the same dimension as the regions")
    if amb != d or any(r.ambient_dimension() != d for r in regions):
        raise C.CsdError(C.CSD_ERR_DIMENSION, f"regions have dimension {amb}, the plant {d}")
    ids = np.ascontiguousarray(np.asarray(list(robot_geometry_ids), np.int32).reshape(-1))
    if ids.size == 0:
        raise ValueError("Robot geometry IDs cannot be empty")
    if not voxel_radius > 0:
        raise ValueError("Voxel radius must be positive")
    v = _voxel_rows(voxels)
    if v.shape[0] > MAX_NUM_VOXELS:
        raise RuntimeError("Voxel buffer size insufficient")
    n = col.shape[1]
    seg = np.ascontiguousarray(np.asarray(list(line_segment_idxs), np.int64).reshape(-1))
    if seg.size != n:
        raise ValueError("one line segment index per collision is required")
    if n and (seg.min() < 0 or seg.max() >= m):
        raise IndexError("line segment index out of range")
    if options.verbose:
        print(f"[EditRegionsCuda] Num collisions to be optimized {n}")
    if n == 0:
        raise RuntimeError("[EditRegionsCuda] No collisions are contained in the regions, this is not supported.\n")
    q = np.ascontiguousarray(col.T)
    seg32 = np.ascontiguousarray(seg.astype(np.uint32))
    A = np.ascontiguousarray(np.concatenate([np.asarray(r.A(), np.float32).reshape(-1, d) for r in regions]))
    b = np.ascontiguousarray(np.concatenate([np.asarray(r.b(), np.float32).reshape(-1) for r in regions]))
    off = np.zeros(m + 1, np.int32)
    off[1:] = np.cumsum([r.b().size for r in regions])
    cap = int(off[-1]) + n
    A_out = np.zeros((cap, d), np.float32)
    b_out = np.zeros(cap, np.float32)
    nf = np.zeros(m, np.int32)
    proj = np.zeros((n, d), np.float32)
    opt = np.zeros((n, d), np.float32)
    o = options._c()
    C.check(C.lib().csd_edit_regions(h.handle, C.ptr(q), C.ptr(seg32), ctypes.c_int64(n),
                                     C.ptr(np.ascontiguousarray(ls.T)), C.ptr(np.ascontiguousarray(le.T)), m,
                                     C.ptr(A), C.ptr(b), C.ptr(off), C.ptr(v) if v.size else None, v.shape[0],
                                     ctypes.c_float(voxel_radius), C.ptr(ids), ids.size, ctypes.byref(o),
                                     C.ptr(A_out), C.ptr(b_out), C.ptr(nf), C.ptr(proj), C.ptr(opt)))
    counts = np.bincount(seg, minlength=m)
    coff = np.concatenate([[0], np.cumsum(counts)])
    edited = []
    for r in range(m):
        if counts[r] == 0:
            if options.verbose:
                print(f"[EditRegionsCuda] region {r} remains unchanged")
            edited.append(regions[r])
            continue
        row = int(off[r] + coff[r])
        if options.verbose:
            print(f"[EditRegionsCuda] region {r} added {int(nf[r]) - regions[r].b().size} faces")
        edited.append(HPolyhedron(A_out[row:row + nf[r]], b_out[row:row + nf[r]]))
    return edited, (np.ascontiguousarray(proj.T), np.ascontiguousarray(opt.T))


class BatchedEdgeInflator:
    """Many EI-ZO inflations advancing together on the GPU (csd_batch_*): each
    slot has its own plant, segment and domain and yields exactly the region
    CudaEdgeInflator.inflateEdge would for the same inputs (no voxels).
    inflate() takes any number of inflations: up to max_slots run at once and
    the rest start in slots as earlier ones finish."""

    SAMPLE_VARIANTS = ("8 face pairs/lane, 1 block/SM", "8 face pairs/lane, 2 blocks/SM",
                       "8 face pairs/lane, 3 blocks/SM", "16 face pairs/lane, 1 block/SM",
                       "16 face pairs/lane, 2 blocks/SM")
    SAMPLE_FLOP_RULE = ("(2 d + 4) F per chain and mixing step: a . dir (2 d), the carried-slack update (2) and the "
                        "two theta-bound compares (2) per face, FMA = 2, division not counted; summed over the slots "
                        "and iterations of the step")
    CHECK_ITEM_CAPS = (8, 16, 32, 128, 512)

    def __init__(self, plants: Sequence[MinimalPlant], options: EizoOptions, max_slots: int,
                 face_capacity: int = MAX_NUM_FACES, autotune_iterations: int = 4):
        self._plants = list(plants)
        self._handles = [plant_handle(p) for p in self._plants]
        self._options = options
        self._capacity = int(face_capacity)
        self._max_slots = int(max_slots)
        arr = (ctypes.c_void_p * len(self._handles))(*[h.handle.value for h in self._handles])
        self._opt_c = options._c()
        h = ctypes.c_void_p()
        C.check(C.lib().csd_batch_create(arr, len(self._handles), self._max_slots, ctypes.byref(self._opt_c),
                                         self._capacity, ctypes.byref(h)))
        self._handle = h
        self.last_iterations = None
        if autotune_iterations:
            self.autotune(autotune_iterations)

    def autotune(self, iterations: int = 4) -> None:
        """Time every sampler variant and check work-item cap on the first
        `iterations` iterations of the next inflate and keep the fastest."""
        C.check(C.lib().csd_batch_autotune(self._handle, int(iterations)))

    def set_surrogate(self, surrogate, stop_probability: float = 0.1) -> None:
        """Surrogate-guided checking with a CollisionSurrogate holding one net
        per plant of this batch (None turns it off)."""
        self._surrogate = surrogate  # keep the bank alive while the batch uses it
        C.check(C.lib().csd_batch_set_surrogate(self._handle, surrogate.handle if surrogate is not None else None,
                                                ctypes.c_float(stop_probability)))

    def set_surrogate_rounds(self, rounds: int, first_round: int) -> None:
        """Round schedule of the surrogate-guided check (see csd_capi.h)."""
        C.check(C.lib().csd_batch_set_surrogate_rounds(self._handle, int(rounds), int(first_round)))

    def set_shapes(self, sample_variant: int, check_item_cap: int) -> None:
        """Fix the sampler variant (index into SAMPLE_VARIANTS) and the check
        work-item cap instead of tuning."""
        C.check(C.lib().csd_batch_set_shapes(self._handle, int(sample_variant), int(check_item_cap)))

    def tuning(self) -> dict:
        sv, cap, nv = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        ms = np.zeros(64, np.float32)
        C.check(C.lib().csd_batch_tuning(self._handle, ctypes.byref(sv), ctypes.byref(cap), C.ptr(ms),
                                         ctypes.byref(nv)))
        ns = len(self.SAMPLE_VARIANTS)
        if nv.value != ns + len(self.CHECK_ITEM_CAPS):
            raise RuntimeError(f"the library reports {nv.value} tuned shapes, the names list "
                               f"{ns} sampler variants + {len(self.CHECK_ITEM_CAPS)} check caps")
        t, lg, lr = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        C.check(C.lib().csd_batch_sample_variants(self._handle, ctypes.byref(t), ctypes.byref(lg), ctypes.byref(lr)))
        return {"sample_variant": self.SAMPLE_VARIANTS[sv.value], "check_item_cap": cap.value,
                "large_region_variant": self.SAMPLE_VARIANTS[lg.value],
                "last_run_variant": self.SAMPLE_VARIANTS[lr.value],
                "sample_ms": dict(zip(self.SAMPLE_VARIANTS, ms[:ns].tolist())),
                "check_ms": dict(zip(self.CHECK_ITEM_CAPS, ms[ns:nv.value].tolist()))}

    def inflate(self, slot_plant: Sequence[int], line_starts: Sequence[np.ndarray], line_ends: Sequence[np.ndarray],
                domains: Sequence[HPolyhedron]) -> List[HPolyhedron]:
        n = len(slot_plant)
        if not (len(line_starts) == len(line_ends) == len(domains) == n):
            raise ValueError("one segment and one domain per slot")
        dims = [self._handles[int(i)].dim for i in slot_plant]
        sp = np.ascontiguousarray(np.asarray(slot_plant, np.int32))
        starts = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float32).reshape(-1) for x in line_starts]))
        ends = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float32).reshape(-1) for x in line_ends]))
        for d, x in zip(dims, line_starts):
            if np.asarray(x).size != d:
                raise RuntimeError("segment dimension does not match the slot's plant")
        A = np.ascontiguousarray(np.concatenate([np.asarray(dm.A(), np.float32).reshape(-1) for dm in domains]))
        b = np.ascontiguousarray(np.concatenate([np.asarray(dm.b(), np.float32).reshape(-1) for dm in domains]))
        off = np.zeros(n + 1, np.int32)
        off[1:] = np.cumsum([dm.A().shape[0] for dm in domains])
        A_out = np.zeros(sum(self._capacity * d for d in dims), np.float32)
        b_out = np.zeros(n * self._capacity, np.float32)
        nf = np.zeros(n, np.int32)
        nit = np.zeros(n, np.int32)
        ms = ctypes.c_float(0)
        C.check(C.lib().csd_batch_inflate(self._handle, n, C.ptr(sp), C.ptr(starts), C.ptr(ends), C.ptr(A), C.ptr(b),
                                          C.ptr(off), C.ptr(A_out), C.ptr(b_out), C.ptr(nf), C.ptr(nit),
                                          ctypes.byref(ms)))
        self.last_iterations = nit
        self.last_device_ms = ms.value
        cfg = np.zeros(n, np.int64)
        C.check(C.lib().csd_batch_configs_checked(self._handle, n, C.ptr(cfg)))
        self.last_configs_checked = cfg
        nl = ctypes.c_int64(0)
        C.check(C.lib().csd_batch_last_launches(self._handle, ctypes.byref(nl)))
        self.last_kernel_launches = int(nl.value)
        out, aoff = [], 0
        for i, d in enumerate(dims):
            Ai = A_out[aoff:aoff + nf[i] * d].reshape(nf[i], d).copy()
            out.append(HPolyhedron(Ai, b_out[i * self._capacity:i * self._capacity + nf[i]].copy()))
            aoff += self._capacity * d
        return out

    STAGES = ("sample", "score", "sort", "check", "compact", "bisect", "faces", "step")

    def set_profiling(self, enable: bool) -> None:
        """Launch stage by stage with events (no graph) and accumulate each
        stage's GPU time; toggling resets the accumulators."""
        C.check(C.lib().csd_batch_set_profiling(self._handle, int(bool(enable))))

    def iteration_profile(self):
        """(stage_ms [iterations, 6], active slots [iterations]) of the last
        inflate in profiling mode."""
        cnt = ctypes.c_int32(0)
        C.check(C.lib().csd_batch_iteration_profile(self._handle, 0, None, None, ctypes.byref(cnt)))
        ms = np.zeros((cnt.value, len(self.STAGES)), np.float32)
        act = np.zeros(cnt.value, np.int32)
        C.check(C.lib().csd_batch_iteration_profile(self._handle, cnt.value, C.ptr(ms), C.ptr(act),
                                                    ctypes.byref(cnt)))
        return ms, act

    def iteration_variants(self):
        """(sampler variant index [iterations], most faces of an active region
        [iterations]) of the last inflate in profiling mode."""
        cnt = ctypes.c_int32(0)
        C.check(C.lib().csd_batch_iteration_variants(self._handle, 0, None, None, ctypes.byref(cnt)))
        var = np.zeros(cnt.value, np.int32)
        faces = np.zeros(cnt.value, np.int32)
        C.check(C.lib().csd_batch_iteration_variants(self._handle, cnt.value, C.ptr(var), C.ptr(faces),
                                                     ctypes.byref(cnt)))
        return var, faces

    def sample_flops(self) -> float:
        """Sampler FLOPs of the last inflate in profiling mode (SAMPLE_FLOP_RULE)."""
        v = ctypes.c_double(0)
        C.check(C.lib().csd_batch_sample_flops(self._handle, ctypes.byref(v)))
        return v.value

    def stage_ms(self) -> dict:
        ms = np.zeros(len(self.STAGES), np.float32)
        C.check(C.lib().csd_batch_stage_ms(self._handle, C.ptr(ms)))
        return dict(zip(self.STAGES, ms.tolist()))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h and C._lib is not None:
            try:
                C._lib.csd_batch_destroy(h)
            except Exception:  # pragma: no cover
                pass
        self._handle = None
