"""Plant loader: the reference parser's grouping, traversal and pair rules."""
import numpy as np

from csdecomp_b200 import scenes
from csdecomp_b200.plant import CollisionGroup, URDFParser


def test_pair_rule_boxes_in_corners(plants):
    p = plants["boxes_in_corners"].plant
    # 4 world boxes x 1 robot sphere; world-world pairs are skipped (urdf_parser.cpp:559)
    assert p.num_collision_pairs == 4
    assert plants["boxes_in_corners"].robot_geometry_ids == [4]


def test_kinova_scene_counts(plants):
    gp = plants["kinova_on_table"]
    assert gp.dim == 7
    assert gp.plant.kin_tree.num_links == 33
    assert gp.plant.num_collision_pairs == 137
    seq = gp.plant.kin_tree.joint_traversal_sequence
    assert sorted(seq.tolist()) == list(range(gp.plant.kin_tree.num_joints))


def test_traversal_is_dfs_from_root(plants):
    kt = plants["2_branch_5dof"].plant.kin_tree
    seen = {0}
    for j in kt.joint_traversal_sequence:
        assert kt.joint_parent_link[j] in seen
        seen.add(int(kt.joint_child_link[j]))


def test_synthetic_scene_is_seeded():
    a = scenes.point_check_scene()
    b = scenes.point_check_scene()
    for k, v in a.plant.arrays().items():
        np.testing.assert_array_equal(v, b.plant.arrays()[k])
    assert a.plant.num_scene_geometries == 60
    groups = [g.group for g in a.plant.scene_collision_geometries]
    assert groups.count(CollisionGroup.WORLD) == 20
    # every robot sphere is paired with every world box
    assert a.plant.num_collision_pairs >= 40 * 20


def test_edge_scene_keepout():
    s = scenes.edge_check_scene(keepout=0.8)
    assert s.plant.num_scene_geometries == 284
    caps = [g for g in s.plant.scene_collision_geometries if g.type == 3]
    assert len(caps) == 4
