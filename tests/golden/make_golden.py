"""Generates the golden fixtures in this directory from the reference's own
test assets and known-answer tests (run where the reference source tree is
available; the fixtures are committed so tests never read it):

    python tests/golden/make_golden.py /root/reference

Outputs
  ref_assets/  the reference's test models as loader fixtures: every
               csdecomp/tests/test_assets/*.urdf and directives/*.yml, copied
               as they are (text only; the meshes they name are not copied,
               the loaders read no meshes)
  plants.npz   plant tables of the reference test robots, parsed from
               csdecomp/tests/test_assets/*.urdf, directives/kinova_sens_on_table.yml
               and the inline URDF of edge_inflation_zero_order_test.cpp:72-115
               with csdecomp_b200.plant.URDFParser (the reference parser's rules)
  golden.json  known answers transcribed from the reference tests (file:line
               beside each entry)
"""
from __future__ import annotations

import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from csdecomp_b200.plant import URDFParser  # noqa: E402

PLANT_KEYS = ("joint_type", "joint_parent_link", "joint_child_link", "joint_idx_to_config_idx",
              "joint_traversal_sequence", "joint_X_PL_J", "joint_axis", "geom_type", "geom_link_index",
              "geom_group", "geom_dimensions", "geom_X_L_B", "collision_pairs_flat")


def raw_urdf_from_test(path: str) -> str:
    src = open(path).read()
    m = re.search(r'R"\((.*?)\)"', src, re.S)
    if not m:
        raise RuntimeError(f"no raw URDF string in {path}")
    return m.group(1)


def dump_plant(out: dict, name: str, parser: URDFParser) -> None:
    mp = parser.get_minimal_plant()
    kt = parser.get_kinematic_tree()
    a = mp.arrays()
    for k in PLANT_KEYS:
        out[f"{name}/{k}"] = a[k]
    out[f"{name}/meta"] = np.array([mp.kin_tree.num_joints, mp.kin_tree.num_links,
                                    mp.kin_tree.num_configuration_variables, mp.num_scene_geometries,
                                    mp.num_collision_pairs], np.int64)
    out[f"{name}/lower"] = kt.getPositionLowerLimits()
    out[f"{name}/upper"] = kt.getPositionUpperLimits()
    out[f"{name}/robot_geometry_ids"] = np.array(parser.get_scene_inspector().robot_geometry_ids, np.int32)
    names = sorted(kt.link_name_to_index.items(), key=lambda kv: kv[1])
    out[f"{name}/link_names"] = np.array([n for n, _ in names])


def copy_assets(assets: str) -> None:
    dst = os.path.join(HERE, "ref_assets")
    os.makedirs(os.path.join(dst, "directives"), exist_ok=True)
    for sub, ext in (("", ".urdf"), ("directives", ".yml")):
        src = os.path.join(assets, sub)
        for f in sorted(os.listdir(src)):
            if f.endswith(ext):
                shutil.copyfile(os.path.join(src, f), os.path.join(dst, sub, f))


def main(ref: str) -> None:
    assets = os.path.join(ref, "csdecomp", "tests", "test_assets")
    copy_assets(assets)
    out: dict = {}
    for name in ("2_branch_5dof", "3dofrobot", "3dofrobot_prismatic", "3dofrobot_spheres", "movable_block"):
        p = URDFParser()
        p.parse_urdf(os.path.join(assets, name + ".urdf"))
        dump_plant(out, name, p)
    p = URDFParser()
    p.register_package("test_assets", assets)
    p.parse_directives(os.path.join(assets, "directives", "kinova_sens_on_table.yml"))
    dump_plant(out, "kinova_on_table", p)
    p = URDFParser()
    p.parse_urdf_string(raw_urdf_from_test(
        os.path.join(ref, "csdecomp", "src", "planning", "tests", "edge_inflation_zero_order_test.cpp")))
    dump_plant(out, "boxes_in_corners", p)
    p = URDFParser()
    p.parse_urdf_string(raw_urdf_from_test(
        os.path.join(ref, "csdecomp", "src", "planning", "tests", "cuda_visibility_graph_test.cpp")))
    dump_plant(out, "vg_boxes", p)
    np.savez_compressed(os.path.join(HERE, "plants.npz"), **out)

    kinova_q = [-2.4934235, -1.6654704, -1.9375235, 1.9090002, 0.09470118]
    golden = {
        "fk": [
            {"src": "csdecomp/src/plant/tests/minimal_kinematic_tree_test.cpp:58-69", "plant": "2_branch_5dof",
             "q": [1, 1, 1, 1, 1], "link": "link1",
             "X": [[0.540302, -0.841471, 0, 0], [0.841471, 0.540302, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]]},
            {"src": "csdecomp/src/plant/tests/minimal_kinematic_tree_test.cpp:71-82", "plant": "2_branch_5dof",
             "q": [1, 1, 1, 1, 1], "link": "link2",
             "X": [[-0.41614684, -0.90929743, 0.0, 0.54030231], [0.90929743, -0.41614684, 0.0, 0.84147098],
                   [0, 0, 1, 0], [0, 0, 0, 1]]},
            {"src": "csdecomp/src/plant/tests/minimal_kinematic_tree_test.cpp:83-89", "plant": "2_branch_5dof",
             "q": [1, 1, 1, 1, 1], "link": "link6",
             "X": [[-0.9899925, -0.14112001, 0.0, -1.0596646], [0.14112001, -0.9899925, 0.0, 0.58067513],
                   [0, 0, 1, 0], [0, 0, 0, 1]]},
            {"src": "csdecomp/src/plant/tests/minimal_kinematic_tree_test.cpp:114-125 and "
                    "cuda_forward_kinematics_test.cpp:29-73", "plant": "3dofrobot_prismatic",
             "q": [1, 1, 1], "link": "link3",
             "X": [[0.60952558, 0.17919833, 0.77224771, 1.75935346], [0.59500984, 0.54030231, -0.59500984, 1.19001968],
                   [-0.52387199, 0.8221687, 0.22270331, -1.88921496], [0, 0, 0, 1]]},
        ],
        "verdicts": [
            {"src": "csdecomp/src/plant/tests/collision_checker_test.cpp:28-41", "plant": "3dofrobot",
             "free": [[0, 1.8, 2.46]], "col": [[0, 1.8, 2.47]]},
            {"src": "csdecomp/src/plant/tests/collision_checker_test.cpp:43-61", "plant": "2_branch_5dof",
             "free": [[0.6714, -0.9096, 0.79, -0.1806, 0.0], [0.0204, 0.3714, 0.4714, 1.0344, -1.2816]],
             "col": [[0.6714, -0.9096, 0.78, -0.1806, 0.0], [0.0204, 0.3714, 0.4714, 1.0874, -1.2816]]},
            {"src": "csdecomp/src/plant/tests/collision_checker_test.cpp:63-75", "plant": "3dofrobot_spheres",
             "free": [[0, 0, 2.67]], "col": [[0, 0, 2.68]]},
            {"src": "csdecomp/src/plant/tests/collision_checker_test.cpp:77-105", "plant": "movable_block",
             "free": np.array([[-0.375, -0.375, 0.004, 0.004, -0.003, -0.002],
                               [-0.622, -0.416, 0.002, 0.04, 0.088, 0.303],
                               [-0.099, -0.099, 0.0, 0.008, 0.008, 0.692],
                               [1.0224, -0.3276, 0.0014, -0.0056, -0.8796, 0.0564],
                               [0.7724, 0.7724, 0.0024, 0.0024, -0.7956, -0.7956]]).T.tolist(),
             "col": np.array([[-0.375, -0.375, -0.002, -0.002, 0.237, 0.591],
                              [-0.461, -0.416, 0.088, 0.088, 0.202, 0.318],
                              [-0.099, -0.099, 0.008, 0.008, 0.592, 0.449],
                              [1.0224, -0.8546, -0.8796, 0.0564, -0.0256, -0.0256],
                              [0.7724, 0.7974, -0.7956, -0.7956, -0.7956, -0.0116]]).T.tolist()},
            {"src": "csdecomp/src/plant/tests/collision_checker_test.cpp:167-196", "plant": "kinova_on_table",
             "free": [[0] * 7, kinova_q + [1.8022158, 1.6754638], kinova_q + [1.8349, 1.6754638]],
             "col": [kinova_q + [1.8679, 1.6754638]]},
        ],
        "voxel_verdicts": {
            "src": "csdecomp/src/plant/tests/collision_checker_test.cpp:107-165 and "
                   "cuda_collision_checker_test.cpp:200-261",
            "plant": "movable_block", "grid": [6, 6, 6], "spacing": [0.3, 0.3, 0.1], "radius": 0.02,
            "free": np.array([[0.00, 0.00, 0.00], [0.00, 0.00, 0.00], [0.00, 0.00, 0.27], [0.00, 0.00, 0.57],
                              [0.00, 1.50, 1.27]]).T.tolist(),
            "col": np.array([[0.15, 0.00, 0.00, 0.00, 0.16], [0.00, 0.15, 0.48, 0.48, 0.28],
                             [0.00, 0.00, 0.00, 0.31, 0.06], [0.00, 0.87, -0.43, -0.43, 1.46],
                             [0.00, 1.17, 1.17, 1.17, 1.59]]).T.tolist()},
        "projection": {"src": "csdecomp/src/planning/tests/cuda_set_builder_utils_test.cpp:19-68",
                       "start": [0, 1], "end": [2, 1.8], "samples": [[0, 0], [3.5, 0], [1.5, 0]],
                       "mid_projection": [0.948276, 1.37931]},
        "visibility_graph": {"src": "csdecomp/src/planning/tests/cuda_visibility_graph_test.cpp:132-152",
                             "plant": "vg_boxes", "step": 0.1,
                             "nodes": [[0, 0], [1.5, 0], [0, 1.5], [-1.5, 0], [0, -1.5]],
                             "adjacency_upper": [1, 1, 1, 1, 0, 1, 0, 0, 1, 0]},
        "eizo_2d": [
            {"src": "csdecomp/src/planning/tests/edge_inflation_zero_order_test.cpp:118-173",
             "start": [0, 0], "end": [1, 0], "inside": [[1.8, 0.2]], "outside": [[1.8, 0.4]], "voxels": [],
             "voxel_radius": 0.01},
            {"src": "csdecomp/src/planning/tests/edge_inflation_zero_order_test.cpp:198-271",
             "start": [-0.5, 0], "end": [0, 0.5], "inside": [[0.0, 0.0]], "outside": [[0.0, 0.8]], "voxels": [],
             "voxel_radius": 0.01},
            {"src": "csdecomp/src/planning/tests/edge_inflation_zero_order_test.cpp:356-430",
             "start": [-0.5, 1.75], "end": [0.5, 1.75], "inside": [[-1.75, 1.75], [1.75, 1.75]], "outside": [],
             "voxels": [], "voxel_radius": 0.01},
            {"src": "csdecomp/src/planning/tests/edge_inflation_zero_order_test.cpp:498-586",
             "start": [-0.5, 1.75], "end": [0.5, 1.75], "inside": [[1.75, 1.8]], "outside": [[-1.75, 1.75]],
             "voxels": [[-0.55, 2.05, 0.0], [-1.50, 1.80, 0.0], [1.90, 1.90, 0.0]], "voxel_radius": 0.05},
        ],
        "eizo_kinova": [
            {"src": "csdecomp/src/planning/tests/edge_inflation_zero_order_test.cpp:432-496",
             "start": [0] * 7, "end": [0, 1, -1, 0.5, 0, 0, 0], "num_particles": 2000, "max_iterations": 100,
             "mixing_steps": 40, "voxels": [], "voxel_radius": 0.01, "frac_bound": 1.2},
        ],
        "eizo_throws": {"src": "csdecomp/src/planning/tests/edge_inflation_zero_order_test.cpp:175-196",
                        "num_particles_too_many": 1000000, "domain_faces": 4000},
        # the test's inline URDF is the one of edge_inflation_zero_order_test.cpp (checked below)
        "edit_regions_2d": {"src": "csdecomp/src/planning/tests/cuda_edit_regions_test.cpp:79-227",
                            "plant": "boxes_in_corners", "configuration_margin": 0.01, "bisection_steps": 9,
                            "voxels": [[-0.55, 2.02, 0.0], [-1.50, 1.80, 0.0], [1.90, 1.90, 0.0]],
                            "voxel_radius": 0.05,
                            "starts": [[-1.90, 0.00], [0.00, 0.00], [0.00, 1.80]],
                            "ends": [[0.00, 0.00], [0.00, 1.80], [1.90, 1.80]],
                            "collisions": [[-0.9, 1.0], [0.6, 0.5], [1.1, -1.0], [1.9, 1.9]],
                            "repeats": 3,
                            "unbisected_steps": 1, "unbisected_col": 1, "unbisected_tol": 1e-6},
    }
    if raw_urdf_from_test(os.path.join(ref, "csdecomp", "src", "planning", "tests", "cuda_edit_regions_test.cpp")) != \
            raw_urdf_from_test(os.path.join(ref, "csdecomp", "src", "planning", "tests",
                                            "edge_inflation_zero_order_test.cpp")):
        raise RuntimeError("cuda_edit_regions_test.cpp no longer uses the boxes_in_corners URDF")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote", os.path.join(HERE, "plants.npz"), "and golden.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_golden.py <root of the reference source tree>")
    main(sys.argv[1])
