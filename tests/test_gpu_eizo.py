"""EI-ZO on the GPU: the reference's 2-D and Kinova tests, replay
bit-exactness against the oracle, and the reference's error cases."""
import numpy as np
import pytest

import csdecomp_b200 as csd
from csdecomp_b200 import scenes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def domain_of(gp):
    d = csd.HPolyhedron()
    d.MakeBox(gp.lower, gp.upper)
    return d


def frac_in_collision(plant, P, start, voxels=None, vr=0.0, rids=(), n=1000):
    s = csd.UniformSampleInHPolyhedraCuda([P], np.asarray(start, np.float32).reshape(-1, 1), n, 50, seed=777)[0]
    if voxels is None:
        return 1.0 - csd.CheckCollisionFreeCuda(s, plant).mean()
    return 1.0 - csd.CheckCollisionFreeVoxelsCuda(s, csd.Voxels(voxels), vr, plant, rids).mean()


@pytest.mark.parametrize("case_idx", range(4))
def test_eizo_2d_golden(plants, golden, case_idx):
    case = golden["eizo_2d"][case_idx]
    gp = plants["boxes_in_corners"]
    opt = csd.EizoOptions(num_particles=1000)
    vox = np.array(case["voxels"], np.float32).reshape(-1, 3).T
    info = csd.EizoInfo()
    mp = csd.EizoCuda(case["start"], case["end"], csd.Voxels(vox), case["voxel_radius"], domain_of(gp), gp.plant,
                      gp.robot_geometry_ids, opt, info)
    P = csd.HPolyhedron(mp)
    assert P.PointInSet(case["start"]) and P.PointInSet(case["end"])
    for x in case["inside"]:
        assert P.PointInSet(x), (case["src"], x)
    for x in case["outside"]:
        assert not P.PointInSet(x), (case["src"], x)
    mid = 0.5 * (np.array(case["start"], np.float32) + np.array(case["end"], np.float32))
    frac = frac_in_collision(gp.plant, P, mid, vox if vox.size else None, case["voxel_radius"],
                             gp.robot_geometry_ids)
    assert frac < opt.epsilon * 1.1
    assert len(info.iteration_info) >= 1


def replay(plant, ls, le, domain, opt, rids=(), voxels=None, vr=0.0):
    """The oracle's EI-ZO driven by GPU verdicts: every downstream step
    (sampling, compaction, projection, bisection, faces) must then match the
    GPU run bit for bit."""
    def checker(q):
        if voxels is None:
            return csd.CheckCollisionFreeCuda(q.T, plant)
        return csd.CheckCollisionFreeVoxelsCuda(q.T, csd.Voxels(voxels), vr, plant, rids)
    vrows = None if voxels is None else np.ascontiguousarray(np.asarray(voxels, np.float32).T)
    return O.eizo(plant, ls, le, domain.A(), domain.b(), opt, rids, vrows, vr, checker=checker)


def test_eizo_replay_bit_exact_2d(plants):
    gp = plants["boxes_in_corners"]
    opt = csd.EizoOptions(num_particles=1000)
    dom = domain_of(gp)
    inf = csd.CudaEdgeInflator(gp.plant, gp.robot_geometry_ids, opt, dom)
    P = inf.inflateEdge([-0.5, 0.0], [0.0, 0.5], None, 0.01, verbose=False)
    A, b, iters = replay(gp.plant, [-0.5, 0.0], [0.0, 0.5], dom, opt)
    np.testing.assert_array_equal(P.A(), A)
    np.testing.assert_array_equal(P.b(), b)
    gi = inf.last_info.iteration_info
    assert [i.num_faces_placed for i in gi] == [r["num_faces_placed"] for r in iters]
    assert [i.num_collisions_unadaptive for i in gi] == [r["num_collisions_unadaptive"] for r in iters]


def test_eizo_replay_bit_exact_7dof():
    sc = scenes.edge_check_scene(keepout=0.8)
    q = sc.random_configs(4000, 17)
    free = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1]
    ls = free[0]
    le = np.clip(ls + 0.15, -np.pi, np.pi).astype(np.float32)
    if not csd.CheckEdgeCollisionFree(ls, le, sc.plant):
        le = ls.copy()
    dom = csd.HPolyhedron()
    dom.MakeBox(sc.lower(), sc.upper())
    opt = csd.EizoOptions(num_particles=500, mixing_steps=20, max_iterations=6)
    inf = csd.CudaEdgeInflator(sc.plant, sc.inspector.robot_geometry_ids, opt, dom)
    P = inf.inflateEdge(ls, le, None, 0.0, verbose=False)
    A, b, _ = replay(sc.plant, ls, le, dom, opt)
    np.testing.assert_array_equal(P.A(), A)
    np.testing.assert_array_equal(P.b(), b)
    assert P.A().shape[0] > 14


def test_eizo_replay_bit_exact_voxels(plants, golden):
    case = golden["eizo_2d"][3]
    gp = plants["boxes_in_corners"]
    vox = np.array(case["voxels"], np.float32).T
    opt = csd.EizoOptions(num_particles=1000)
    dom = domain_of(gp)
    inf = csd.CudaEdgeInflator(gp.plant, gp.robot_geometry_ids, opt, dom)
    P = inf.inflateEdge(case["start"], case["end"], csd.Voxels(vox), case["voxel_radius"], verbose=False)
    A, b, _ = replay(gp.plant, case["start"], case["end"], dom, opt, gp.robot_geometry_ids, vox,
                     case["voxel_radius"])
    np.testing.assert_array_equal(P.A(), A)
    np.testing.assert_array_equal(P.b(), b)


def test_eizo_kinova(plants, golden):
    case = golden["eizo_kinova"][0]
    gp = plants["kinova_on_table"]
    opt = csd.EizoOptions(num_particles=case["num_particles"], max_iterations=case["max_iterations"])
    mp = csd.EizoCuda(case["start"], case["end"], None, 0.01, domain_of(gp), gp.plant, gp.robot_geometry_ids, opt)
    P = csd.HPolyhedron(mp)
    assert P.PointInSet(case["start"]) and P.PointInSet(case["end"])
    mid = 0.5 * (np.array(case["start"], np.float32) + np.array(case["end"], np.float32))
    assert frac_in_collision(gp.plant, P, mid) < opt.epsilon * case["frac_bound"]


def test_eizo_throws(plants, golden):
    gp = plants["boxes_in_corners"]
    opt = csd.EizoOptions(num_particles=golden["eizo_throws"]["num_particles_too_many"])
    with pytest.raises(RuntimeError):
        csd.EizoCuda([0, 0], [1, 0], None, 0.01, domain_of(gp), gp.plant, gp.robot_geometry_ids, opt)
    n = golden["eizo_throws"]["domain_faces"]
    dom2 = csd.HPolyhedron(np.zeros((n, 2), np.float32), np.zeros(n, np.float32))
    with pytest.raises(RuntimeError):
        csd.EizoCuda([0, 0], [1, 0], None, 0.01, dom2, gp.plant, gp.robot_geometry_ids,
                     csd.EizoOptions(num_particles=10))


def test_inflator_is_deterministic_and_reusable(plants):
    gp = plants["boxes_in_corners"]
    inf = csd.CudaEdgeInflator(gp.plant, gp.robot_geometry_ids, csd.EizoOptions(num_particles=800), domain_of(gp))
    a = inf.inflateEdge([0, 0], [1, 0], None, 0.01, verbose=False)
    b = inf.inflateEdge([-0.5, 1.75], [0.5, 1.75], None, 0.01, verbose=False)
    c = inf.inflateEdge([0, 0], [1, 0], None, 0.01, verbose=False)
    np.testing.assert_array_equal(a.A(), c.A())
    assert not np.array_equal(a.A(), b.A()) or a.A().shape != b.A().shape


def test_points_post_bisection_2d(plants):
    """EizoIterationInfo.points_post_bisection (kept for dim <= 3 with
    track_iteration_information, as the reference does): dim x K points,
    K = num_collisions_updated, every one in collision."""
    gp = plants["boxes_in_corners"]
    opt = csd.EizoOptions(num_particles=500, track_iteration_information=True)
    inf = csd.CudaEdgeInflator(gp.plant, gp.robot_geometry_ids, opt, domain_of(gp))
    inf.inflateEdge([-0.5, 0.0], [0.0, 0.5], None, 0.01, verbose=False)
    its = inf.last_info.iteration_info
    placed = [it for it in its if it.num_collisions_updated > 0]
    assert placed
    for it in placed:
        pts = it.points_post_bisection
        assert pts.shape == (2, it.num_collisions_updated)
        assert not csd.CheckCollisionFreeCuda(pts, gp.plant).any()
    assert its[-1].points_post_bisection.size == 0 or its[-1].num_collisions_updated > 0
    opt.track_iteration_information = False
    inf = csd.CudaEdgeInflator(gp.plant, gp.robot_geometry_ids, opt, domain_of(gp))
    inf.inflateEdge([-0.5, 0.0], [0.0, 0.5], None, 0.01, verbose=False)
    assert all(it.points_post_bisection.size == 0 for it in inf.last_info.iteration_info)
