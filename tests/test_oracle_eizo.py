"""EI-ZO on the CPU oracle against the reference's 2-D tests
(edge_inflation_zero_order_test.cpp:118-430, 498-586) -- no GPU."""
import numpy as np
import pytest

from oracle import oracle as O
from csdecomp_b200.api import EizoOptions


def box_domain(lo, hi):
    d = len(lo)
    A = np.zeros((2 * d, d), np.float32)
    b = np.zeros(2 * d, np.float32)
    for i in range(d):
        A[2 * i, i], A[2 * i + 1, i] = -1, 1
        b[2 * i], b[2 * i + 1] = -lo[i], hi[i]
    return A, b


def frac_in_collision(plant, A, b, start, vox, vr, rids, n=1000):
    s, nf = O.hit_and_run(A, b, start, n, 50, seed=99, stream=5)
    assert nf == 0
    return 1.0 - O.check_points(plant, s, O.RULE_GPU, vox if len(vox) else None, vr, rids).mean()


@pytest.mark.parametrize("case_idx", range(4))
def test_eizo_2d_golden(plants, golden, case_idx):
    case = golden["eizo_2d"][case_idx]
    gp = plants["boxes_in_corners"]
    A0, b0 = box_domain(gp.lower, gp.upper)
    opt = EizoOptions(num_particles=1000)
    vox = np.array(case["voxels"], np.float32).reshape(-1, 3)
    A, b, iters = O.eizo(gp.plant, case["start"], case["end"], A0, b0, opt, gp.robot_geometry_ids,
                         vox if len(vox) else None, case["voxel_radius"])
    inside = lambda x: bool(np.all(A @ np.asarray(x, np.float32) <= b + 1e-6))
    assert inside(case["start"]) and inside(case["end"])
    for x in case["inside"]:
        assert inside(x), (case["src"], x)
    for x in case["outside"]:
        assert not inside(x), (case["src"], x)
    mid = 0.5 * (np.array(case["start"], np.float32) + np.array(case["end"], np.float32))
    frac = frac_in_collision(gp.plant, A, b, mid, vox, case["voxel_radius"], gp.robot_geometry_ids)
    assert frac < opt.epsilon * 1.1
    assert iters[-1]["num_collisions_unadaptive"] <= iters[-1]["collisions_threshold"] + 1


def test_eizo_faces_separate_their_collisions(plants):
    gp = plants["boxes_in_corners"]
    A0, b0 = box_domain(gp.lower, gp.upper)
    opt = EizoOptions(num_particles=1000)
    A, b, _ = O.eizo(gp.plant, [0, 0], [1, 0], A0, b0, opt, gp.robot_geometry_ids)
    assert A.shape[0] > A0.shape[0]
    np.testing.assert_allclose(np.linalg.norm(A[A0.shape[0]:], axis=1), 1.0, atol=1e-5)


def test_eizo_does_not_depend_on_the_thread_count(plants):
    """The oracle is the parity checker: its regions must not depend on how
    many host threads run its point checks."""
    gp = plants["boxes_in_corners"]
    A0, b0 = box_domain(gp.lower, gp.upper)
    opt = EizoOptions(num_particles=500)
    A1, b1, it1 = O.eizo(gp.plant, [0, 0], [1, 0], A0, b0, opt, gp.robot_geometry_ids, nthreads=1)
    A4, b4, it4 = O.eizo(gp.plant, [0, 0], [1, 0], A0, b0, opt, gp.robot_geometry_ids, nthreads=4)
    np.testing.assert_array_equal(A1, A4)
    np.testing.assert_array_equal(b1, b4)
    assert it1 == it4


def test_eizo_face_capacity_exceeded_raises(plants):
    gp = plants["boxes_in_corners"]
    A0, b0 = box_domain(gp.lower, gp.upper)
    opt = EizoOptions(num_particles=500)
    A, _, _ = O.eizo(gp.plant, [0, 0], [1, 0], A0, b0, opt, gp.robot_geometry_ids)
    assert A.shape[0] - A0.shape[0] >= 2
    with pytest.raises(RuntimeError, match="Max face count exceeded"):
        O.eizo(gp.plant, [0, 0], [1, 0], A0, b0, opt, gp.robot_geometry_ids, capacity=A0.shape[0] + 1)
