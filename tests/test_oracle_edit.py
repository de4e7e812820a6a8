"""EditRegionsCuda on the CPU oracle against the reference's own test
(cuda_edit_regions_test.cpp:79-227) -- no GPU."""
import numpy as np
import pytest

from oracle import oracle as O


def box_domain(lo, hi):
    d = len(lo)
    A = np.zeros((2 * d, d), np.float32)
    b = np.zeros(2 * d, np.float32)
    for i in range(d):
        A[2 * i, i], A[2 * i + 1, i] = -1, 1
        b[2 * i], b[2 * i + 1] = -lo[i], hi[i]
    return A, b


def point_in_set(A, b, x, tol=1e-9):
    """hpolyhedron.cpp:265-274 in FP32."""
    return bool(np.all(A @ np.asarray(x, np.float32) <= b + np.float32(tol)))


def golden_case(plants, golden, steps=None):
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    dom = box_domain(gp.lower, gp.upper)
    col = np.array(g["collisions"], np.float32)
    rep = np.tile(col, (g["repeats"], 1))
    seg = np.repeat(np.arange(g["repeats"], dtype=np.uint32), len(col))
    out = O.edit_regions(gp.plant, rep, seg, g["starts"], g["ends"], [dom] * len(g["starts"]),
                         gp.robot_geometry_ids, g["voxels"], g["voxel_radius"], g["configuration_margin"],
                         g["bisection_steps"] if steps is None else steps)
    return g, col, rep, seg, out


def test_edit_regions_golden(plants, golden):
    g, col, rep, seg, (regions, proj, opt) = golden_case(plants, golden)
    assert proj.shape == opt.shape == rep.shape
    for r, (A, b) in enumerate(regions):
        assert point_in_set(A, b, g["starts"][r]) and point_in_set(A, b, g["ends"][r])
        for x in opt:
            assert not point_in_set(A, b, x)
        for x in col:
            assert not point_in_set(A, b, x)
        # faces beyond the domain's four are unit normals
        np.testing.assert_allclose(np.linalg.norm(A[4:], axis=1), 1.0, atol=1e-5)


def test_edit_regions_unbisected_keeps_collision(plants, golden):
    g, col, rep, seg, (regions, proj, opt) = golden_case(plants, golden, steps=golden["edit_regions_2d"]["unbisected_steps"])
    c = g["unbisected_col"]
    assert np.linalg.norm(opt[c] - col[c]) <= g["unbisected_tol"]


def test_edit_regions_grouping_and_projection(plants, golden):
    """Collisions given out of segment order come back grouped (stable), with
    their projections on their own segment."""
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    dom = box_domain(gp.lower, gp.upper)
    col = np.array(g["collisions"], np.float32)
    seg = np.array([2, 0, 2, 1], np.uint32)
    regions, proj, opt = O.edit_regions(gp.plant, col, seg, g["starts"], g["ends"], [dom] * 3,
                                        gp.robot_geometry_ids, g["voxels"], g["voxel_radius"], 0.01, 0)
    order = np.argsort(seg, kind="stable")
    np.testing.assert_array_equal(opt, col[order])  # zero bisection steps keep the collisions
    for i, j in enumerate(order):
        s = np.array(g["starts"][seg[j]], np.float32)
        e = np.array(g["ends"][seg[j]], np.float32)
        t = np.clip(np.dot(col[j] - s, e - s) / np.dot(e - s, e - s), 0, 1)
        np.testing.assert_allclose(proj[i], s + t * (e - s), atol=1e-6)


def test_edit_regions_region_without_collisions_unchanged(plants, golden):
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    dom = box_domain(gp.lower, gp.upper)
    col = np.array(g["collisions"], np.float32)
    seg = np.zeros(len(col), np.uint32)
    regions, _, _ = O.edit_regions(gp.plant, col, seg, g["starts"], g["ends"], [dom] * 3,
                                   gp.robot_geometry_ids, g["voxels"], g["voxel_radius"])
    for A, b in regions[1:]:
        np.testing.assert_array_equal(A, dom[0])
        np.testing.assert_array_equal(b, dom[1])
    assert regions[0][0].shape[0] > 4


def test_edit_regions_collision_outside_region_adds_no_face(plants, golden):
    """A collision outside its region is skipped (cuda_edit_regions.cu:253-259)."""
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    A = np.array([[-1, 0], [1, 0], [0, -1], [0, 1]], np.float32)
    b = np.array([1.95, 0.1, 0.1, 0.1], np.float32)  # a thin box around segment 0 only
    col = np.array([[0.6, 0.5]], np.float32)
    regions, _, _ = O.edit_regions(gp.plant, col, [0], [g["starts"][0]], [g["ends"][0]], [(A, b)],
                                   gp.robot_geometry_ids, g["voxels"], g["voxel_radius"])
    np.testing.assert_array_equal(regions[0][0], A)


def test_edit_regions_bad_segment_index(plants, golden):
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    dom = box_domain(gp.lower, gp.upper)
    with pytest.raises(RuntimeError):
        O.edit_regions(gp.plant, [[0.6, 0.5]], [3], g["starts"], g["ends"], [dom] * 3, gp.robot_geometry_ids)


def test_edit_regions_does_not_depend_on_the_thread_count(plants, golden):
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    dom = box_domain(gp.lower, gp.upper)
    col = np.tile(np.array(g["collisions"], np.float32), (g["repeats"], 1))
    seg = np.repeat(np.arange(g["repeats"], dtype=np.uint32), len(g["collisions"]))
    outs = [O.edit_regions(gp.plant, col, seg, g["starts"], g["ends"], [dom] * len(g["starts"]),
                           gp.robot_geometry_ids, g["voxels"], g["voxel_radius"], g["configuration_margin"],
                           g["bisection_steps"], nthreads=t) for t in (1, 4)]
    (r1, p1, o1), (r4, p4, o4) = outs
    np.testing.assert_array_equal(p1, p4)
    np.testing.assert_array_equal(o1, o4)
    for (A1, b1), (A4, b4) in zip(r1, r4):
        np.testing.assert_array_equal(A1, A4)
        np.testing.assert_array_equal(b1, b4)
