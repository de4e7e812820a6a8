"""ctypes wrapper around liboracle.so -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's CPU/GPU algorithms on the CPU (see
csd_oracle.cpp for the file:line each function follows). It is the checker:
only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference arms may import this module; the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

RULE_CPU, RULE_GPU = 0, 1
EDGE_L2_REF, EDGE_LINF, EDGE_VG = 0, 1, 2

_P = ctypes.c_void_p


class OrcPlant(ctypes.Structure):
    _fields_ = [
        ("num_joints", ctypes.c_int32),
        ("num_links", ctypes.c_int32),
        ("num_configuration_variables", ctypes.c_int32),
        ("num_geometries", ctypes.c_int32),
        ("num_collision_pairs", ctypes.c_int32),
        ("joint_type", _P),
        ("joint_parent_link", _P),
        ("joint_child_link", _P),
        ("joint_idx_to_config_idx", _P),
        ("joint_traversal_sequence", _P),
        ("joint_X_PL_J", _P),
        ("joint_axis", _P),
        ("geom_type", _P),
        ("geom_link_index", _P),
        ("geom_group", _P),
        ("geom_dimensions", _P),
        ("geom_X_L_B", _P),
        ("collision_pairs_flat", _P),
    ]


class OrcEizoOptions(ctypes.Structure):
    _fields_ = [
        ("configuration_margin", ctypes.c_float),
        ("tau", ctypes.c_float),
        ("delta", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("bisection_steps", ctypes.c_uint32),
        ("num_particles", ctypes.c_uint32),
        ("max_hyperplanes_per_iteration", ctypes.c_uint32),
        ("max_iterations", ctypes.c_uint32),
        ("mixing_steps", ctypes.c_uint32),
        ("seed", ctypes.c_uint64),
    ]


class OrcEizoIter(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "iteration_index", "num_samples_drawn", "collisions_threshold",
        "num_collisions_unadaptive", "num_collisions_updated", "num_faces_placed")]


CHECKER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                              ctypes.c_void_p)


def build() -> str:
    """Compile liboracle.so with oracle/Makefile (g++ only, no CUDA)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_edge_num_points.restype = ctypes.c_int64
        _lib.orc_num_samples_unadaptive.restype = ctypes.c_uint32
        _lib.orc_num_samples_unadaptive.argtypes = [ctypes.c_float] * 3
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class PlantView:
    """Keeps the plant's arrays alive while the oracle holds pointers to them."""

    def __init__(self, plant):
        self.arrays: Dict[str, np.ndarray] = plant.arrays()
        kt = plant.kin_tree
        a = self.arrays
        self.s = OrcPlant(kt.num_joints, kt.num_links, kt.num_configuration_variables,
                          plant.num_scene_geometries, plant.num_collision_pairs,
                          *[_ptr(a[k]) for k in (
                              "joint_type", "joint_parent_link", "joint_child_link",
                              "joint_idx_to_config_idx", "joint_traversal_sequence", "joint_X_PL_J",
                              "joint_axis", "geom_type", "geom_link_index", "geom_group",
                              "geom_dimensions", "geom_X_L_B", "collision_pairs_flat")])
        self.dim = kt.num_configuration_variables
        self.num_links = kt.num_links

    @property
    def ref(self):
        return ctypes.byref(self.s)


def _configs(q: np.ndarray, dim: int) -> np.ndarray:
    q = np.ascontiguousarray(q, np.float32)
    return q.reshape(-1, dim)


def fk(plant, q: np.ndarray, fp64: bool = False) -> np.ndarray:
    pv = PlantView(plant)
    qq = _configs(q, pv.dim)
    n = qq.shape[0]
    out = np.zeros((n, pv.num_links, 16), np.float64 if fp64 else np.float32)
    f = lib().orc_fk_f64 if fp64 else lib().orc_fk_f32
    f(pv.ref, _ptr(qq), ctypes.c_int64(n), _ptr(out))
    return out


def _vox(voxels, robot_ids):
    if voxels is None or len(voxels) == 0:
        return None, 0, None, 0
    v = np.ascontiguousarray(np.asarray(voxels, np.float32).reshape(-1, 3))
    r = np.ascontiguousarray(np.asarray(robot_ids, np.int32).reshape(-1))
    return v, v.shape[0], r, r.shape[0]


def check_points(plant, q: np.ndarray, rule: int = RULE_GPU, voxels=None, voxel_radius: float = 0.0,
                 robot_geometry_ids: Sequence[int] = (), nthreads: int = 0) -> np.ndarray:
    pv = PlantView(plant)
    qq = _configs(q, pv.dim)
    n = qq.shape[0]
    out = np.zeros(n, np.uint8)
    v, nv, r, nr = _vox(voxels, robot_geometry_ids)
    rc = lib().orc_check_points(pv.ref, _ptr(qq), ctypes.c_int64(n), rule, _ptr(v), nv,
                                ctypes.c_float(voxel_radius), _ptr(r), nr, _ptr(out), nthreads)
    if rc:
        raise RuntimeError(f"oracle point check failed ({rc})")
    return out


def signed_distance(plant, q: np.ndarray, voxels=None, voxel_radius: float = 0.0,
                    robot_geometry_ids: Sequence[int] = (), nthreads: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """(FP64 verdict, minimum signed distance over pairs) per configuration."""
    pv = PlantView(plant)
    qq = _configs(q, pv.dim)
    n = qq.shape[0]
    ver = np.zeros(n, np.uint8)
    sd = np.zeros(n, np.float64)
    v, nv, r, nr = _vox(voxels, robot_geometry_ids)
    rc = lib().orc_signed_distance_f64(pv.ref, _ptr(qq), ctypes.c_int64(n), _ptr(v), nv,
                                       ctypes.c_float(voxel_radius), _ptr(r), nr, _ptr(ver), _ptr(sd),
                                       nthreads)
    if rc:
        raise RuntimeError(f"oracle signed distance failed ({rc})")
    return ver, sd


def check_edges(plant, starts: np.ndarray, ends: np.ndarray, step: float = 0.01, mode: int = EDGE_L2_REF,
                rule: int = RULE_GPU, nthreads: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    pv = PlantView(plant)
    s = _configs(starts, pv.dim)
    e = _configs(ends, pv.dim)
    n = s.shape[0]
    out = np.zeros(n, np.uint8)
    pts = np.zeros(n, np.int64)
    rc = lib().orc_check_edges(pv.ref, _ptr(s), _ptr(e), ctypes.c_int64(n), ctypes.c_float(step), mode, rule,
                               _ptr(out), _ptr(pts), nthreads)
    if rc:
        raise RuntimeError(f"oracle edge check failed ({rc})")
    return out, pts


def edge_num_points(q1, q2, step: float, mode: int) -> int:
    a = np.ascontiguousarray(q1, np.float32)
    b = np.ascontiguousarray(q2, np.float32)
    return int(lib().orc_edge_num_points(_ptr(a), _ptr(b), a.size, ctypes.c_float(step), mode))


def edge_points(q1, q2, step: float, mode: int) -> np.ndarray:
    a = np.ascontiguousarray(q1, np.float32)
    b = np.ascontiguousarray(q2, np.float32)
    n = edge_num_points(a, b, step, mode)
    out = np.zeros((n, a.size), np.float32)
    for k in range(n):
        lib().orc_edge_point(_ptr(a), _ptr(b), a.size, ctypes.c_float(step), mode, ctypes.c_int64(k),
                             _ptr(out[k]))
    return out


def pair_collision_free(ga, X_W_LA, gb, X_W_LB, rule: int = RULE_CPU) -> int:
    def g(x):
        return (int(x.type), np.ascontiguousarray(x.dimensions, np.float32),
                np.ascontiguousarray(np.asarray(x.X_L_B, np.float32).T.reshape(-1)))
    ta, da, xa = g(ga)
    tb, db, xb = g(gb)
    wa = np.ascontiguousarray(np.asarray(X_W_LA, np.float32).T.reshape(-1))
    wb = np.ascontiguousarray(np.asarray(X_W_LB, np.float32).T.reshape(-1))
    return int(lib().orc_pair_collision_free(ta, _ptr(da), _ptr(xa), _ptr(wa), tb, _ptr(db), _ptr(xb),
                                             _ptr(wb), rule))


def hit_and_run(A: np.ndarray, b: np.ndarray, x0: np.ndarray, num_samples: int, mixing_steps: int,
                seed: int = 1337, stream: int = 0, nthreads: int = 0) -> Tuple[np.ndarray, int]:
    A = np.ascontiguousarray(A, np.float32)
    b = np.ascontiguousarray(b, np.float32).reshape(-1)
    x0 = np.ascontiguousarray(x0, np.float32).reshape(-1)
    F, d = A.shape
    out = np.zeros((num_samples, d), np.float32)
    nf = ctypes.c_int32(0)
    rc = lib().orc_hit_and_run(_ptr(A), _ptr(b), F, d, _ptr(x0), num_samples, mixing_steps,
                               ctypes.c_uint64(seed), ctypes.c_uint32(stream), _ptr(out), ctypes.byref(nf),
                               nthreads)
    if rc:
        raise RuntimeError("oracle hit-and-run failed")
    return out, nf.value


def rng_direction(seed: int, chain: int, stream: int, step: int, dim: int) -> np.ndarray:
    out = np.zeros(dim + 1, np.float32)
    lib().orc_rng_direction(ctypes.c_uint64(seed), ctypes.c_uint32(chain), ctypes.c_uint32(stream),
                            ctypes.c_uint32(step), dim, _ptr(out))
    return out


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(o))
    return o


def num_samples_unadaptive(epsilon: float, delta: float, tau: float) -> int:
    return int(lib().orc_num_samples_unadaptive(epsilon, delta, tau))


def eizo(plant, line_start, line_end, A_domain, b_domain, options, robot_geometry_ids=(), voxels=None,
         voxel_radius: float = 0.0, capacity: int = 4000, checker=None, nthreads: int = 0):
    """CPU EI-ZO. ``checker(q[n,d]) -> uint8[n]`` replaces the oracle's own
    point check when given (used to replay GPU verdicts through the oracle's
    downstream steps). Returns (A, b, iteration records)."""
    pv = PlantView(plant)
    d = pv.dim
    A = np.zeros((capacity, d), np.float32)
    b = np.zeros(capacity, np.float32)
    F0 = np.asarray(A_domain).shape[0]
    A[:F0] = A_domain
    b[:F0] = np.asarray(b_domain).reshape(-1)
    nf = ctypes.c_int32(F0)
    o = OrcEizoOptions(options.configuration_margin, options.tau, options.delta, options.epsilon,
                       options.bisection_steps, options.num_particles, options.max_hyperplanes_per_iteration,
                       options.max_iterations, options.mixing_steps, options.seed)
    iters = (OrcEizoIter * max(1, int(options.max_iterations)))()
    nit = ctypes.c_int32(0)
    v, nv, r, nr = _vox(voxels, robot_geometry_ids)
    cb = None
    if checker is not None:
        def _cb(qp, n, outp, ctx):
            try:
                qa = np.ctypeslib.as_array(ctypes.cast(qp, ctypes.POINTER(ctypes.c_float)), shape=(n * d,))
                res = np.asarray(checker(qa.reshape(n, d).copy()), np.uint8)
                oa = np.ctypeslib.as_array(ctypes.cast(outp, ctypes.POINTER(ctypes.c_uint8)), shape=(n,))
                oa[:] = res
                return 0
            except Exception:  # pragma: no cover - surfaced as an error code
                return 1
        cb = CHECKER_FN(_cb)
    ls = np.ascontiguousarray(line_start, np.float32)
    le = np.ascontiguousarray(line_end, np.float32)
    rc = lib().orc_eizo(pv.ref, _ptr(ls), _ptr(le), _ptr(v), nv, ctypes.c_float(voxel_radius), _ptr(r), nr,
                        ctypes.byref(o), _ptr(A), _ptr(b), ctypes.byref(nf), capacity, cb, None, iters,
                        ctypes.byref(nit), nthreads)
    if rc == 2:
        raise RuntimeError("Max face count exceeded.")
    if rc:
        raise RuntimeError(f"oracle eizo failed ({rc})")
    recs = [dict((k, getattr(iters[i], k)) for k, _ in OrcEizoIter._fields_) for i in range(nit.value)]
    return A[:nf.value].copy(), b[:nf.value].copy(), recs


def _checker_cb(checker, d):
    if checker is None:
        return None

    def _cb(qp, n, outp, ctx):
        try:
            qa = np.ctypeslib.as_array(ctypes.cast(qp, ctypes.POINTER(ctypes.c_float)), shape=(n * d,))
            res = np.asarray(checker(qa.reshape(n, d).copy()), np.uint8)
            oa = np.ctypeslib.as_array(ctypes.cast(outp, ctypes.POINTER(ctypes.c_uint8)), shape=(n,))
            oa[:] = res
            return 0
        except Exception:  # pragma: no cover - surfaced as an error code
            return 1
    return CHECKER_FN(_cb)


def edit_regions(plant, collisions, line_segment_idxs, starts, ends, regions, robot_geometry_ids=(), voxels=None,
                 voxel_radius: float = 0.0, configuration_margin: float = 0.01, bisection_steps: int = 9,
                 checker=None, nthreads: int = 0):
    """CPU EditRegionsCuda (cuda_edit_regions.cu:44-301). collisions [n][d]
    with one segment index each; starts/ends [m][d]; regions a list of (A, b).
    ``checker(q[n,d]) -> uint8[n]`` replaces the oracle's own point check when
    given. Returns ([(A, b)] per region, projections [n][d], optimized [n][d]),
    the last two in the grouped (segment-stable) order the reference returns."""
    pv = PlantView(plant)
    d = pv.dim
    c = np.ascontiguousarray(np.asarray(collisions, np.float32).reshape(-1, d))
    n = c.shape[0]
    seg = np.ascontiguousarray(np.asarray(line_segment_idxs, np.uint32).reshape(-1))
    ls = np.ascontiguousarray(np.asarray(starts, np.float32).reshape(-1, d))
    le = np.ascontiguousarray(np.asarray(ends, np.float32).reshape(-1, d))
    m = ls.shape[0]
    A = np.ascontiguousarray(np.concatenate([np.asarray(a, np.float32).reshape(-1, d) for a, _ in regions]))
    b = np.ascontiguousarray(np.concatenate([np.asarray(bb, np.float32).reshape(-1) for _, bb in regions]))
    off = np.zeros(m + 1, np.int32)
    off[1:] = np.cumsum([np.asarray(bb).size for _, bb in regions])
    cap = int(off[-1]) + n
    A_out = np.zeros((max(cap, 1), d), np.float32)
    b_out = np.zeros(max(cap, 1), np.float32)
    nf = np.zeros(m, np.int32)
    proj = np.zeros((max(n, 1), d), np.float32)
    opt = np.zeros((max(n, 1), d), np.float32)
    if voxels is not None and len(voxels):
        v = np.ascontiguousarray(np.asarray(voxels, np.float32).reshape(-1, 3))
    else:
        v = None
    r = np.ascontiguousarray(np.asarray(robot_geometry_ids, np.int32).reshape(-1))
    rc = lib().orc_edit_regions(pv.ref, _ptr(c), _ptr(seg), ctypes.c_int64(n), _ptr(ls), _ptr(le), m, _ptr(A),
                                _ptr(b), _ptr(off), _ptr(v), 0 if v is None else v.shape[0],
                                ctypes.c_float(voxel_radius), _ptr(r), r.size, ctypes.c_float(configuration_margin),
                                ctypes.c_uint32(bisection_steps), _ptr(A_out), _ptr(b_out), _ptr(nf), _ptr(proj),
                                _ptr(opt), _checker_cb(checker, d), None, nthreads)
    if rc:
        raise RuntimeError(f"oracle edit_regions failed ({rc})")
    counts = np.bincount(seg, minlength=m) if n else np.zeros(m, np.int64)
    coff = np.concatenate([[0], np.cumsum(counts)])
    out = []
    for i in range(m):
        row = int(off[i] + coff[i])
        out.append((A_out[row:row + nf[i]].copy(), b_out[row:row + nf[i]].copy()))
    return out, proj[:n].copy(), opt[:n].copy()
