"""Plant loader: the reference parser's grouping, traversal and pair rules."""
import numpy as np
import pytest

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


def test_plant_wrapper(plants):
    """Plant (minimal_plant.h:42-145) over the parser's outputs gives the
    parser's MinimalPlant and the reference's accessors."""
    import os
    from csdecomp_b200.plant import Plant, URDFParser
    d = os.path.join(os.path.dirname(__file__), "golden", "loader")
    p = URDFParser()
    p.register_package("loader_assets", d)
    p.parse_directives(os.path.join(d, "cell.yml"))
    pl = Plant(p.get_kinematic_tree(), p.get_scene_inspector(), p.get_scene_collision_geometries())
    a = p.get_minimal_plant().arrays()
    b = pl.getMinimalPlant().arrays()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert pl.numLinks() == 10 and pl.numJoints() == 9 and pl.numConfigurationVariables() == 3
    assert pl.getRobotGeometryIds() == p.get_scene_inspector().robot_geometry_ids
    names = pl.getSceneCollisionGeometryNames()
    assert len(names) == len(p.get_scene_collision_geometries())
    for i, n in enumerate(names):
        assert pl.getSceneCollisionGeometryIndexByName(n) == i
    with pytest.raises(IndexError):
        pl.getSceneCollisionGeometryIndexByName("no such geometry")
    np.testing.assert_array_equal(pl.getCollisionPairMatrix(), p.get_scene_inspector().get_collision_pair_matrix())


def test_minimal_tree_structs(plants):
    """MinimalJoint / MinimalLink views agree with the tables."""
    kt = plants["kinova_on_table"].plant.kin_tree
    joints, links = kt.joints, kt.links
    assert len(joints) == kt.num_joints and len(links) == kt.num_links
    for j in joints:
        assert links[j.child_link].parent_joint_index == j.index
        assert j.index in links[j.parent_link].child_joint_index_array
    assert links[0].parent_joint_index == -1
    assert sum(l.num_child_joints for l in links) == kt.num_joints


def test_tree_accessors(plants):
    """KinematicTree and URDFParser accessors of plant_bindings.h:14-63."""
    import os
    d = os.path.join(os.path.dirname(__file__), "golden", "loader")
    p = URDFParser()
    p.register_package("loader_assets", d)
    p.parse_directives(os.path.join(d, "cell.yml"))
    kt = p.get_kinematic_tree()
    assert kt.is_finalized()
    i = kt.get_link_index("arm::upper")
    assert kt.get_link_name(i) == "arm::upper" and kt.get_link(i).name == "arm::upper"
    j = kt.get_joint_index("arm::elbow")
    assert j >= 0 and kt.get_joint(j).name == "arm::elbow" and kt.get_joint_index("nope") == -1
    assert len(kt.get_links()) == 10 and len(kt.get_joints()) == 9
    leaves = kt.get_leaf_link_indices()
    assert all(not kt.get_link(l).child_joints for l in leaves)
    assert kt.get_link_index("post::pole") in leaves
    with pytest.raises(ValueError):
        kt.compute_link_frame_to_world_transforms(np.zeros(2))
    pl = p.build_plant()
    np.testing.assert_array_equal(pl.getMinimalPlant().arrays()["geom_type"], p.get_minimal_plant().arrays()["geom_type"])
    p2 = URDFParser()
    with pytest.raises(RuntimeError):
        p2.build_plant()
