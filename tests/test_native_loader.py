"""The library's C++ model loader (csd_urdf_*, the reference's URDFParser for
C++ callers) against the Python loader, whose tables the golden fixtures pin:
identical MinimalPlant tables, robot geometry ids, limits and geometry names
on generated URDFs, on the directives fixture in tests/golden/loader, and on
the reference's own test models (tests/golden/ref_assets, copied there by
tests/golden/make_golden.py); the same errors on malformed models. No GPU is
used."""
import os

import numpy as np
import pytest

from csdecomp_b200 import _capi as C
from csdecomp_b200.plant import URDFParser

HERE = os.path.dirname(os.path.abspath(__file__))
LOADER = os.path.join(HERE, "golden", "loader")
REF_ASSETS = os.path.join(HERE, "golden", "ref_assets")  # the reference's test models (make_golden.py)


def assert_same(py: URDFParser, nat: C.NativeURDFParser):
    a = py.get_minimal_plant().arrays()
    b, dim, L = nat.arrays()
    assert set(a) == set(b)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    kt = py.get_kinematic_tree()
    assert dim == kt.num_configuration_variables and L == len(kt.links)
    assert nat.robot_geometry_ids() == py.get_scene_inspector().robot_geometry_ids
    lo, hi = nat.position_limits()
    np.testing.assert_array_equal(lo, kt.getPositionLowerLimits())
    np.testing.assert_array_equal(hi, kt.getPositionUpperLimits())
    for name, idx in py.get_scene_inspector().scene_collision_geometry_name_to_geometry_index.items():
        assert nat.geometry_index(name) == idx, name
    for name, idx in kt.link_name_to_index.items():
        assert nat.link_index(name) == idx, name


def random_urdf(seed: int) -> str:
    """A random tree (revolute, prismatic and fixed joints, rotated origins,
    boxes, spheres and capsules, named and unnamed collisions, links without
    geometry, limits present or absent) attached to the world."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 12))
    out = [f'<robot name="r{seed}">']

    def origin(p=0.8):
        if rng.random() > p:
            return ""
        xyz = " ".join(f"{v:.7g}" for v in rng.uniform(-0.5, 0.5, 3))
        rpy = " ".join(f"{v:.9g}" for v in rng.uniform(-3.2, 3.2, 3))
        return f'<origin xyz="{xyz}" rpy="{rpy}"/>' if rng.random() < 0.7 else f'<origin xyz="{xyz}"/>'
    for i in range(n):
        out.append(f'<link name="l{i}">')
        for c in range(int(rng.integers(0, 4))):
            kind = rng.integers(0, 3)
            if kind == 0:
                shape = '<box size="{:.6g} {:.6g} {:.6g}"/>'.format(*rng.uniform(0.01, 0.4, 3))
            elif kind == 1:
                shape = f'<sphere radius="{rng.uniform(0.01, 0.2):.6g}"/>'
            else:
                shape = f'<capsule radius="{rng.uniform(0.01, 0.1):.6g}" length="{rng.uniform(0.05, 0.5):.6g}"/>'
            name = f' name="c{i}_{c}"' if rng.random() < 0.5 else ""
            out.append(f"<collision{name}>{origin()}<geometry>{shape}</geometry></collision>")
        out.append("</link>")
    parents = ["world"] + [f"l{int(rng.integers(0, i))}" for i in range(1, n)]
    for i in range(n):
        jt = ["fixed", "revolute", "prismatic"][int(rng.choice(3, p=[0.25, 0.55, 0.2]))]
        body = origin(0.9) + f'<parent link="{parents[i]}"/><child link="l{i}"/>'
        if jt != "fixed":
            body += '<axis xyz="{:.5g} {:.5g} {:.5g}"/>'.format(*rng.normal(size=3))
            if rng.random() < 0.8:
                lo = rng.uniform(-3, 0)
                body += f'<limit lower="{lo:.8g}" upper="{lo + rng.uniform(0.1, 3):.8g}"/>'
        out.append(f'<joint name="j{i}" type="{jt}">{body}</joint>')
    out.append("</robot>")
    return "\n".join(out)


@pytest.mark.parametrize("seed", range(40))
def test_generated_urdf(seed):
    text = random_urdf(seed)
    py, nat = URDFParser(), C.NativeURDFParser()
    py.parse_urdf_string(text)
    nat.parse_urdf_string(text)
    assert_same(py, nat)


def test_directives_fixture():
    py, nat = URDFParser(), C.NativeURDFParser()
    for p in (py, nat):
        assert p.register_package("loader_assets", LOADER)
    assert not nat.register_package("missing", os.path.join(LOADER, "no_such_dir"))
    py.parse_directives(os.path.join(LOADER, "cell.yml"))
    nat.parse_directives(os.path.join(LOADER, "cell.yml"))
    assert_same(py, nat)
    a, dim, L = nat.arrays()
    assert dim == 3 and L == 10  # world, mount, 4 arm links, 2 gripper links, post frame, post
    assert nat.geometry_index("arm::elbow & pad::2") == 2  # entity decoded, collision counter per link


def test_reference_assets():
    """Every URDF and directives file of the reference's test assets: same
    tables, or the same error (most single-model URDFs are not welded to the
    world, which both loaders reject)."""
    cases = [("urdf", os.path.join(REF_ASSETS, f)) for f in sorted(os.listdir(REF_ASSETS)) if f.endswith(".urdf")]
    ddir = os.path.join(REF_ASSETS, "directives")
    cases += [("yml", os.path.join(ddir, f)) for f in sorted(os.listdir(ddir)) if f.endswith(".yml")]
    parsed = 0
    for kind, path in cases:
        py, nat = URDFParser(), C.NativeURDFParser()
        for p in (py, nat):
            p.register_package("test_assets", REF_ASSETS)
        run_py = py.parse_directives if kind == "yml" else py.parse_urdf
        run_nat = nat.parse_directives if kind == "yml" else nat.parse_urdf
        try:
            run_py(path)
        except RuntimeError as e:
            with pytest.raises(ValueError) as ei:
                run_nat(path)
            assert str(e)[:40] == str(ei.value)[:40], path
            continue
        run_nat(path)
        assert_same(py, nat)
        parsed += 1
    assert parsed >= 8


BAD = {
    "duplicate link": '<robot><link name="a"/><link name="a"/></robot>',
    "duplicate joint": ('<robot><link name="a"/><link name="b"/>'
                        '<joint name="j" type="fixed"><parent link="world"/><child link="a"/></joint>'
                        '<joint name="j" type="fixed"><parent link="a"/><child link="b"/></joint></robot>'),
    "joint type": ('<robot><link name="a"/><joint name="j" type="continuous"><parent link="world"/>'
                   '<child link="a"/><axis xyz="0 0 1"/></joint></robot>'),
    "axis": '<robot><link name="a"/><joint name="j" type="revolute"><parent link="world"/><child link="a"/></joint></robot>',
    "cylinder": ('<robot><link name="a"><collision><geometry><cylinder radius="1" length="1"/></geometry></collision>'
                 '</link><joint name="j" type="fixed"><parent link="world"/><child link="a"/></joint></robot>'),
    "not connected": '<robot><link name="a"/><link name="b"/><joint name="j" type="fixed"><parent link="a"/><child link="b"/></joint></robot>',
    "unlinked branch": ('<robot><link name="a"/><link name="b"/>'
                        '<joint name="j" type="fixed"><parent link="world"/><child link="a"/></joint></robot>'),
    "unknown link": '<robot><link name="a"/><joint name="j" type="fixed"><parent link="world"/><child link="z"/></joint></robot>',
    "origin without xyz": ('<robot><link name="a"/><joint name="j" type="fixed"><origin rpy="0 0 1"/>'
                           '<parent link="world"/><child link="a"/></joint></robot>'),
}


@pytest.mark.parametrize("case", sorted(BAD))
def test_errors_match(case):
    text = BAD[case]
    with pytest.raises(RuntimeError) as e_py:
        URDFParser().parse_urdf_string(text)
    with pytest.raises(ValueError) as e_nat:
        C.NativeURDFParser().parse_urdf_string(text)
    assert str(e_py.value)[:30] == str(e_nat.value)[:30]


def test_not_a_robot():
    assert URDFParser().parse_urdf_string("<model/>") is False
    with pytest.raises(ValueError, match="not 'robot'"):
        C.NativeURDFParser().parse_urdf_string("<model/>")
    with pytest.raises(ValueError, match="XML parse error"):
        C.NativeURDFParser().parse_urdf_string("<robot><link name='a'></robot>")
