"""ctypes binding of libcsdecomp_b200.so (declared in include/csd_capi.h).

The library is the product: this module raises if it has not been built
(there is no CPU fallback).
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcsdecomp_b200.so")

CSD_OK, CSD_ERR_INVALID, CSD_ERR_CAPACITY, CSD_ERR_NOT_CONTAINED, CSD_ERR_CUDA, CSD_ERR_UNSUPPORTED, \
    CSD_ERR_DIMENSION, CSD_ERR_NO_DEVICE = range(8)
CSD_PTR_HOST, CSD_PTR_DEVICE = 0, 1
CSD_EDGE_L2_REF, CSD_EDGE_LINF, CSD_EDGE_VG = 0, 1, 2

_P = ctypes.c_void_p


class PlantDesc(ctypes.Structure):
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


class PlantInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "dim", "num_links", "num_fk_joints", "num_moving", "num_static", "num_tile_pairs",
        "num_generic_pairs", "always_colliding")]


class EizoOptionsC(ctypes.Structure):
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
        ("verbose", ctypes.c_int32),
        ("track_iteration_information", ctypes.c_int32),
    ]


class EizoIterC(ctypes.Structure):
    _fields_ = [
        ("iteration_index", ctypes.c_int32),
        ("num_samples_drawn", ctypes.c_int32),
        ("collisions_threshold", ctypes.c_int32),
        ("num_collisions_unadaptive", ctypes.c_int32),
        ("num_collisions_updated", ctypes.c_int32),
        ("num_faces_placed", ctypes.c_int32),
        ("iteration_time_ms", ctypes.c_float),
    ]


class EditRegionsOptionsC(ctypes.Structure):
    _fields_ = [("configuration_margin", ctypes.c_float), ("bisection_steps", ctypes.c_uint32)]


# every entry point declared in include/csd_capi.h
EXPORTS = (
    "csd_last_error", "csd_version", "csd_plant_create", "csd_plant_destroy", "csd_plant_info", "csd_plant_status", "csd_plant_wait_selftest", "csd_fk",
    "csd_check_points", "csd_check_edges", "csd_check_edges_ranked", "csd_visibility_graph", "csd_pair_collision_free", "csd_uniform_sample_hpolyhedra",
    "csd_inflator_create", "csd_inflator_inflate", "csd_inflator_points_post_bisection", "csd_inflator_destroy", "csd_eizo", "csd_eizo_noalloc", "csd_edit_regions", "csd_batch_create", "csd_batch_inflate", "csd_batch_configs_checked",
    "csd_batch_set_profiling", "csd_batch_stage_ms", "csd_batch_iteration_profile", "csd_batch_iteration_variants", "csd_batch_sample_flops", "csd_batch_last_launches",
    "csd_batch_autotune", "csd_batch_tuning", "csd_batch_set_shapes", "csd_batch_sample_variants", "csd_batch_shape_counts", "csd_batch_set_surrogate",
    "csd_batch_set_surrogate_rounds",    "csd_batch_destroy",
    "csd_num_samples_unadaptive", "csd_fp32_fma_probe", "csd_plant_flops", "csd_plant_set_culling",
    "csd_plant_set_voxel_grid",
    "csd_urdf_create", "csd_urdf_destroy", "csd_urdf_register_package", "csd_urdf_parse_file",
    "csd_urdf_parse_string", "csd_urdf_parse_directives", "csd_urdf_plant_desc", "csd_urdf_limits",
    "csd_urdf_robot_geometry_ids", "csd_urdf_link_index", "csd_urdf_geometry_index",
    "csd_mlp_num_params", "csd_mlp_create", "csd_mlp_destroy", "csd_mlp_get_params", "csd_mlp_set_params",
    "csd_mlp_infer", "csd_mlp_gradients", "csd_mlp_train", "csd_mlp_gemm_test",
)

_lib = None


class CsdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: the CUDA library has not been built "
                "(run `python -c 'import __graft_entry__; __graft_entry__.build()'`).")
        L = ctypes.CDLL(LIB_PATH)
        L.csd_last_error.restype = ctypes.c_char_p
        L.csd_num_samples_unadaptive.restype = ctypes.c_uint32
        L.csd_num_samples_unadaptive.argtypes = [ctypes.c_float] * 3
        L.csd_batch_shape_counts.restype = None
        for name in EXPORTS:
            f = getattr(L, name)
            if name not in ("csd_last_error", "csd_num_samples_unadaptive", "csd_batch_shape_counts"):
                f.restype = ctypes.c_int32
        _lib = L
    return _lib


def check(code: int) -> None:
    if code == CSD_OK:
        return
    msg = lib().csd_last_error().decode(errors="replace")
    if code == CSD_ERR_INVALID:
        raise ValueError(msg)
    raise CsdError(code, msg)


def ptr(a) -> ctypes.c_void_p:
    if a is None:
        return None
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    return a.ctypes.data_as(ctypes.c_void_p)


class PlantHandle:
    """Device-resident plant tables (csd_plant_create / csd_plant_destroy)."""

    def __init__(self, arrays: Dict[str, np.ndarray], num_joints: int, num_links: int, dim: int,
                 num_geoms: int, num_pairs: int):
        self._arrays = arrays
        d = PlantDesc(num_joints, num_links, dim, num_geoms, num_pairs,
                      *[ptr(arrays[k]) for k in (
                          "joint_type", "joint_parent_link", "joint_child_link", "joint_idx_to_config_idx",
                          "joint_traversal_sequence", "joint_X_PL_J", "joint_axis", "geom_type",
                          "geom_link_index", "geom_group", "geom_dimensions", "geom_X_L_B",
                          "collision_pairs_flat")])
        h = ctypes.c_void_p()
        check(lib().csd_plant_create(ctypes.byref(d), ctypes.byref(h)))
        self.handle = h
        self.dim = dim
        self.num_links = num_links

    def set_culling(self, enable: bool) -> None:
        """Link-level broad phase of the collision checks on (default) or off."""
        check(lib().csd_plant_set_culling(self.handle, int(bool(enable))))

    def set_voxel_grid(self, enable: bool) -> None:
        """Voxel hash grid of the voxel checks on (default) or off (every voxel tested)."""
        check(lib().csd_plant_set_voxel_grid(self.handle, int(bool(enable))))

    def flops(self) -> dict:
        fk, pl, pa = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().csd_plant_flops(self.handle, ctypes.byref(fk), ctypes.byref(pl), ctypes.byref(pa)))
        return {"fk": fk.value, "placement": pl.value, "pairs": pa.value,
                "total": fk.value + pl.value + pa.value}

    def info(self) -> dict:
        i = PlantInfo()
        check(lib().csd_plant_info(self.handle, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in PlantInfo._fields_}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h and _lib is not None:
            try:
                _lib.csd_plant_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
        self.handle = None


class NativeURDFParser:
    """URDFParser (urdf_parser.h:18-163) run by the library's C++ loader
    (csd_urdf_*): the same tables as csdecomp_b200.plant.URDFParser, without
    Python's XML and YAML modules. For C++ callers the C ABI is the interface;
    this class exposes it to Python for testing and scripting."""

    def __init__(self):
        h = ctypes.c_void_p()
        check(lib().csd_urdf_create(ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.csd_urdf_destroy(h)
            self._h = None

    def register_package(self, name: str, path: str) -> bool:
        ok = ctypes.c_int32(0)
        check(lib().csd_urdf_register_package(self._h, name.encode(), path.encode(), ctypes.byref(ok)))
        return bool(ok.value)

    def parse_urdf(self, path: str) -> bool:
        check(lib().csd_urdf_parse_file(self._h, path.encode()))
        return True

    def parse_urdf_string(self, text: str) -> bool:
        check(lib().csd_urdf_parse_string(self._h, text.encode()))
        return True

    def parse_directives(self, path: str) -> bool:
        check(lib().csd_urdf_parse_directives(self._h, path.encode()))
        return True

    def arrays(self) -> Tuple[Dict[str, np.ndarray], int, int]:
        """(flat tables as MinimalPlant.arrays() gives them, dim, num_links)."""
        d = PlantDesc()
        check(lib().csd_urdf_plant_desc(self._h, ctypes.byref(d)))
        J, G, P = d.num_joints, d.num_geometries, d.num_collision_pairs

        def grab(p, n, ct, dt):
            if n == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(n,)).astype(dt).copy()
        i32, f32 = (ctypes.c_int32, np.int32), (ctypes.c_float, np.float32)
        a = {
            "joint_type": grab(d.joint_type, J, *i32), "joint_parent_link": grab(d.joint_parent_link, J, *i32),
            "joint_child_link": grab(d.joint_child_link, J, *i32),
            "joint_idx_to_config_idx": grab(d.joint_idx_to_config_idx, J, *i32),
            "joint_traversal_sequence": grab(d.joint_traversal_sequence, J, *i32),
            "joint_X_PL_J": grab(d.joint_X_PL_J, 16 * J, *f32), "joint_axis": grab(d.joint_axis, 3 * J, *f32),
            "geom_type": grab(d.geom_type, G, *i32), "geom_link_index": grab(d.geom_link_index, G, *i32),
            "geom_group": grab(d.geom_group, G, *i32), "geom_dimensions": grab(d.geom_dimensions, 3 * G, *f32),
            "geom_X_L_B": grab(d.geom_X_L_B, 16 * G, *f32),
            "collision_pairs_flat": grab(d.collision_pairs_flat, 2 * P, *i32),
        }
        return a, d.num_configuration_variables, d.num_links

    def get_minimal_plant(self):
        from .plant import MinimalPlant
        a, dim, L = self.arrays()
        return MinimalPlant.from_arrays(a, dim, L)

    def robot_geometry_ids(self) -> List[int]:
        p = ctypes.POINTER(ctypes.c_int32)()
        n = ctypes.c_int32(0)
        check(lib().csd_urdf_robot_geometry_ids(self._h, ctypes.byref(p), ctypes.byref(n)))
        return [int(p[i]) for i in range(n.value)]

    def position_limits(self) -> Tuple[np.ndarray, np.ndarray]:
        d = PlantDesc()
        check(lib().csd_urdf_plant_desc(self._h, ctypes.byref(d)))
        lo = np.zeros(d.num_configuration_variables, np.float32)
        hi = np.zeros(d.num_configuration_variables, np.float32)
        check(lib().csd_urdf_limits(self._h, ptr(lo), ptr(hi)))
        return lo, hi

    def link_index(self, name: str) -> int:
        i = ctypes.c_int32(-1)
        check(lib().csd_urdf_link_index(self._h, name.encode(), ctypes.byref(i)))
        return i.value

    def geometry_index(self, name: str) -> int:
        i = ctypes.c_int32(-1)
        check(lib().csd_urdf_geometry_index(self._h, name.encode(), ctypes.byref(i)))
        return i.value
