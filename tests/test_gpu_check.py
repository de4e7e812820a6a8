"""GPU parity of FK, point checks, edge checks and pair tests against the
oracle (through the C ABI)."""
import numpy as np
import pytest

import csdecomp_b200 as csd
from csdecomp_b200 import scenes
from csdecomp_b200.plant import CollisionGeometry, ShapePrimitive
from oracle import oracle as O

pytestmark = pytest.mark.gpu

BAND = 1e-5  # metres: verdicts may differ only within this signed-distance band


def test_golden_verdicts(plants, golden):
    for case in golden["verdicts"]:
        p = plants[case["plant"]].plant
        assert csd.CheckCollisionFreeCuda(np.array(case["free"], np.float32).T, p).all(), case["src"]
        assert not csd.CheckCollisionFreeCuda(np.array(case["col"], np.float32).T, p).any(), case["src"]
        assert csd.CheckCollisionFree(np.array(case["free"][0], np.float32), p)


def test_golden_voxel_verdicts(plants, golden):
    case = golden["voxel_verdicts"]
    gp = plants[case["plant"]]
    nx, ny, nz = case["grid"]
    sx, sy, sz = case["spacing"]
    off = np.array([-(nx - 1) * sx / 2, -(ny - 1) * sy / 2, 0], np.float32)
    vox = np.array([np.array([ix * sx, iy * sy, iz * sz], np.float32) + off
                    for ix in range(nx) for iy in range(ny) for iz in range(nz)], np.float32).T
    f = csd.CheckCollisionFreeVoxelsCuda(np.array(case["free"], np.float32).T, csd.Voxels(vox), case["radius"],
                                         gp.plant, gp.robot_geometry_ids)
    c = csd.CheckCollisionFreeVoxelsCuda(np.array(case["col"], np.float32).T, csd.Voxels(vox), case["radius"],
                                         gp.plant, gp.robot_geometry_ids)
    assert f.all() and not c.any()


@pytest.mark.parametrize("idx", range(4))
def test_fk_golden(plants, golden, idx):
    g = golden["fk"][idx]
    gp = plants[g["plant"]]
    tf = csd.ComputeForwardKinematicsCuda(np.array(g["q"], np.float32).reshape(-1, 1), gp.plant)[0]
    np.testing.assert_allclose(tf[gp.link(g["link"])], np.array(g["X"]), atol=2e-6)
    stacked = csd.computeLinkFrameToWorldTransformsMinimal(np.array(g["q"], np.float32), gp.plant.kin_tree)
    np.testing.assert_allclose(stacked[4 * gp.link(g["link"]):4 * gp.link(g["link"]) + 4], np.array(g["X"]), atol=2e-6)


@pytest.mark.parametrize("name", ["kinova_on_table", "2_branch_5dof", "movable_block", "synthetic14"])
def test_fk_vs_fp64(plants, name):
    if name == "synthetic14":
        sc = scenes.arm_scene(7, num_spheres=40, arms=2)
        p, q = sc.plant, sc.random_configs(3000, 1)
    else:
        gp = plants[name]
        rng = np.random.default_rng(0)
        p = gp.plant
        lo, hi = np.maximum(gp.lower, -np.pi), np.minimum(gp.upper, np.pi)
        q = (lo + (hi - lo) * rng.random((3000, gp.dim))).astype(np.float32)
    tf = csd.ComputeForwardKinematicsCuda(q.T, p)
    ref = O.fk(p, q, fp64=True).reshape(q.shape[0], -1, 4, 4).transpose(0, 1, 3, 2)
    scale = max(1.0, np.abs(ref[..., :3, 3]).max())
    err = np.abs(tf - ref).max()
    # FP32 relative error bound of the FK transforms against the FP64 oracle
    assert err <= 1e-5 * scale, err


def band_parity(plant, q, voxels=None, vr=0.0, rids=()):
    if voxels is None:
        gpu = csd.CheckCollisionFreeCuda(q.T, plant)
    else:
        gpu = csd.CheckCollisionFreeVoxelsCuda(q.T, csd.Voxels(np.asarray(voxels).T), vr, plant, rids)
    ref = O.check_points(plant, q, O.RULE_GPU, voxels, vr, rids)
    v64, sd = O.signed_distance(plant, q, voxels, vr, rids)
    outside = np.abs(sd) > BAND
    assert (gpu[outside] == ref[outside]).all(), np.nonzero(gpu[outside] != ref[outside])
    assert (gpu[outside] == v64[outside]).all()
    return gpu, int((~outside).sum())


@pytest.mark.parametrize("n", [1, 31, 33, 5000])
def test_point_check_sizes(n):
    sc = scenes.point_check_scene()
    band_parity(sc.plant, sc.random_configs(n, 5))


def test_point_check_parity_large():
    sc = scenes.point_check_scene()
    gpu, band = band_parity(sc.plant, sc.random_configs(40000, 11))
    assert 0.1 < gpu.mean() < 0.5
    assert band < 40


def test_point_check_capsules_boxes_spheres():
    sc = scenes.edge_check_scene(keepout=0.8)
    band_parity(sc.plant, sc.random_configs(6000, 3))


def test_point_check_two_arms():
    sc = scenes.arm_scene(21, num_spheres=60, num_capsules=4, num_world_boxes=30, num_world_spheres=30, arms=2,
                          keepout=0.6)
    band_parity(sc.plant, sc.random_configs(4000, 4))


def test_point_check_kinova(plants):
    gp = plants["kinova_on_table"]
    rng = np.random.default_rng(8)
    q = (gp.lower + (gp.upper - gp.lower) * rng.random((8000, gp.dim))).astype(np.float32)
    band_parity(gp.plant, q)


def test_voxels_random(plants):
    gp = plants["movable_block"]
    rng = np.random.default_rng(2)
    q = (gp.lower + (gp.upper - gp.lower) * rng.random((3000, gp.dim))).astype(np.float32)
    vox = rng.uniform(-1, 1, (500, 3)).astype(np.float32)
    band_parity(gp.plant, q, vox, 0.02, gp.robot_geometry_ids)


def voxel_verdicts(plant, q, vox, vr, rids, grid):
    h = csd.plant_handle(plant)
    h.set_voxel_grid(grid)
    try:
        return csd.CheckCollisionFreeVoxelsCuda(q.T, csd.Voxels(vox.T), vr, plant, rids)
    finally:
        h.set_voxel_grid(True)


@pytest.mark.parametrize("case", ["arm_spheres_capsules", "movable_block_boxes", "kinova"])
def test_voxel_grid_matches_every_voxel(plants, case):
    """The voxel hash grid only prunes: verdicts equal the every-voxel sweep
    bit for bit, over voxel clouds of 64 to 20000 voxels (dense near the
    robot, sparse far away), and agree with the oracle outside the band."""
    rng = np.random.default_rng({"arm_spheres_capsules": 1, "movable_block_boxes": 2, "kinova": 3}[case])
    if case == "arm_spheres_capsules":
        sc = scenes.edge_check_scene(keepout=0.8)
        plant, rids, dim = sc.plant, sc.inspector.robot_geometry_ids, sc.dim
        q = sc.random_configs(6000, 9)
    else:
        gp = plants["movable_block" if case == "movable_block_boxes" else "kinova_on_table"]
        plant, rids, dim = gp.plant, gp.robot_geometry_ids, gp.dim
        q = (gp.lower + (gp.upper - gp.lower) * rng.random((6000, gp.dim))).astype(np.float32)
    q = np.concatenate([q, np.full((3, dim), np.nan, np.float32)])  # NaN poses collide in both forms
    mixed = 0
    for nv, vr in [(64, 0.05), (3000, 0.02), (20000, 0.01)]:
        near = rng.normal(0, 0.4, (nv // 2, 3))
        far = rng.uniform(-2.5, 2.5, (nv - nv // 2, 3))
        vox = np.concatenate([near, far]).astype(np.float32)
        on = voxel_verdicts(plant, q, vox, vr, rids, True)
        off = voxel_verdicts(plant, q, vox, vr, rids, False)
        np.testing.assert_array_equal(on, off)
        assert not on[-3:].any()
        mixed += 0 < on[:-3].mean() < 1
    assert mixed >= 1
    band_parity(plant, q[:1500], vox, vr, rids)


def test_nan_configurations_collide():
    """A NaN configuration collides (every pair test of the reference's rule
    fails on NaN), with the link-level broad phase on and off."""
    sc = scenes.edge_check_scene(keepout=0.8)
    h = csd.plant_handle(sc.plant)
    q = sc.random_configs(64, 3)
    q[::4, 2] = np.nan
    for cull in (True, False):
        h.set_culling(cull)
        v = csd.CheckCollisionFreeCuda(q.T, sc.plant)
        assert not v[::4].any(), cull
    h.set_culling(True)
    ref = O.check_points(sc.plant, q[::4], O.RULE_GPU)
    assert not ref.any()


def test_device_robot_ids_refused(plants):
    """csd_check_points reads robot_geometry_ids on the host: a device pointer
    there is refused with CSD_ERR_INVALID, not dereferenced."""
    import ctypes
    import torch
    from csdecomp_b200 import _capi as C
    gp = plants["movable_block"]
    h = csd.plant_handle(gp.plant)
    q = torch.zeros((4, gp.dim), dtype=torch.float32, device="cuda")
    vox = torch.zeros((100, 3), dtype=torch.float32, device="cuda")
    ids = torch.tensor(gp.robot_geometry_ids, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.uint8, device="cuda")
    rc = C.lib().csd_check_points(h.handle, C.ptr(q.data_ptr()), ctypes.c_int64(4), C.ptr(vox.data_ptr()), 100,
                                  ctypes.c_float(0.01), C.ptr(ids.data_ptr()), ids.numel(), C.ptr(out.data_ptr()),
                                  C.CSD_PTR_DEVICE, None)
    assert rc == C.CSD_ERR_INVALID


def test_empty_batch():
    sc = scenes.point_check_scene()
    assert csd.CheckCollisionFreeCuda(np.zeros((7, 0), np.float32), sc.plant).shape == (0,)


@pytest.mark.parametrize("mode", [csd.CSD_EDGE_L2_REF, csd.CSD_EDGE_LINF, csd.CSD_EDGE_VG])
def test_edges_vs_oracle(mode):
    sc = scenes.edge_check_scene(keepout=0.8)
    rng = np.random.default_rng(mode)
    # short edges so that free edges exist
    s = sc.random_configs(1500, 40 + mode)
    e = (s + rng.normal(0, 0.15, s.shape)).astype(np.float32)
    gpu, pts = csd.CheckEdgesCollisionFreeCuda(s.T, e.T, sc.plant, 0.01, mode, return_points_checked=True)
    ref, _ = O.check_edges(sc.plant, s, e, 0.01, mode)
    diff = np.nonzero(gpu != ref)[0]
    # a differing edge must contain a point within the contact band
    for i in diff:
        pts_i = O.edge_points(s[i], e[i], 0.01, mode)
        _, sd = O.signed_distance(sc.plant, pts_i)
        assert np.abs(sd).min() <= BAND, i
    assert len(diff) <= 3
    assert 0.05 < gpu.mean() < 0.95
    n_all = np.array([O.edge_num_points(s[i], e[i], 0.01, mode) for i in range(len(s))])
    assert (pts <= n_all).all() and (pts[gpu == 1] == n_all[gpu == 1]).all()


def test_edge_visibility_graph_golden(plants, golden):
    case = golden["visibility_graph"]
    gp = plants[case["plant"]]
    nodes = np.array(case["nodes"], np.float32)
    n = len(nodes)
    s, e = zip(*[(nodes[i], nodes[j]) for i in range(n - 1) for j in range(i + 1, n)])
    v = csd.CheckEdgesCollisionFreeCuda(np.array(s).T, np.array(e).T, gp.plant, case["step"], csd.CSD_EDGE_VG)
    assert list(v) == case["adjacency_upper"]
    # the all-pairs entry point (VisibilityGraph) gives the same upper triangle
    A = csd.VisibilityGraph(nodes.T, gp.plant, case["step"])
    iu, ju = np.triu_indices(n, 1)
    assert list(np.asarray(A[iu, ju]).ravel()) == case["adjacency_upper"]
    assert A.shape == (n, n) and np.tril(A.toarray()).sum() == 0


@pytest.mark.parametrize("n", [2, 3, 97, 700])
def test_visibility_graph_matches_explicit_edges(n):
    """Edges generated on the device from node pairs equal the same edges
    passed explicitly (every pair i < j, visibility-graph discretisation)."""
    sc = scenes.edge_check_scene(keepout=0.8)
    q = sc.random_configs(4 * n, 11 + n)
    nodes = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1][:n]
    nodes = np.concatenate([nodes, q[:max(0, n - len(nodes))]])  # pad with any configurations
    A = csd.VisibilityGraph(nodes.T, sc.plant, 0.05)
    iu, ju = np.triu_indices(n, 1)
    ref = csd.CheckEdgesCollisionFreeCuda(nodes[iu].T, nodes[ju].T, sc.plant, 0.05, csd.CSD_EDGE_VG)
    np.testing.assert_array_equal(np.asarray(A[iu, ju]).ravel(), ref)
    if n > 3:
        assert 0 < ref.sum() < len(ref)


def test_visibility_graph_rejects_bad_arguments():
    sc = scenes.point_check_scene()
    q = sc.random_configs(3, 1)
    with pytest.raises(ValueError):
        csd.VisibilityGraph(q[:1].T, sc.plant, 0.01)
    with pytest.raises(ValueError):
        csd.VisibilityGraph(q.T, sc.plant, 0.0)


def test_zero_length_edge_reference_rule():
    sc = scenes.point_check_scene()
    q = sc.random_configs(64, 9)
    col = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 0][:1]
    # the reference's rule checks no point on a zero-length edge (collision_checker.cpp:44-52)
    assert csd.CheckEdgesCollisionFreeCuda(col.T, col.T, sc.plant, 0.01, csd.CSD_EDGE_L2_REF)[0] == 1
    assert csd.CheckEdgesCollisionFreeCuda(col.T, col.T, sc.plant, 0.01, csd.CSD_EDGE_LINF)[0] == 0


def test_pair_collision_free_vs_oracle():
    rng = np.random.default_rng(1)
    types = [ShapePrimitive.SPHERE, ShapePrimitive.BOX, ShapePrimitive.CAPSULE]
    agree = 0
    for k in range(60):
        ga = CollisionGeometry(type=types[k % 3], dimensions=np.array([0.3, 0.4, 0.2], np.float32))
        gb = CollisionGeometry(type=types[(k // 3) % 3], dimensions=np.array([0.25, 0.3, 0.35], np.float32))
        if ga.type == ShapePrimitive.SPHERE:
            ga.dimensions[1:] = -1
        if gb.type == ShapePrimitive.SPHERE:
            gb.dimensions[1:] = -1
        Xa = np.eye(4, dtype=np.float32)
        Xb = np.eye(4, dtype=np.float32)
        Xb[:3, :3] = scenes.random_rotation(rng)
        Xb[:3, 3] = rng.uniform(-0.8, 0.8, 3)
        g = csd.PairCollisionFree(ga, Xa, gb, Xb)
        o = O.pair_collision_free(ga, Xa, gb, Xb, O.RULE_GPU)
        agree += int(g == bool(o))
    assert agree >= 59


def test_errors():
    sc = scenes.point_check_scene()
    with pytest.raises(RuntimeError):
        csd.CheckCollisionFreeCuda(np.zeros((5, 3), np.float32), sc.plant)
    with pytest.raises(ValueError):
        csd.CheckCollisionFreeVoxelsCuda(np.zeros((7, 3), np.float32), csd.Voxels(np.zeros((3, 2))), 0.1, sc.plant,
                                         [10 ** 6])
    bad = scenes.point_check_scene()
    bad.plant.scene_collision_geometries[0].type = ShapePrimitive.CYLINDER
    bad.plant._arrays = None
    with pytest.raises(csd.CsdError) as ei:
        csd.CheckCollisionFreeCuda(np.zeros((7, 1), np.float32), bad.plant)
    assert ei.value.code == 5


@pytest.mark.parametrize("arms", [1, 2])
def test_broad_phase_leaves_every_verdict_unchanged(arms):
    """The link-level broad phase only skips pairs whose bounding spheres are
    more than 1e-4 m apart, so verdicts with it on and off are identical."""
    sc = scenes.arm_scene(77 + arms, num_spheres=60, num_capsules=4, num_world_boxes=120, num_world_spheres=120,
                          arms=arms, keepout=0.6, arm_spacing=1.4)
    q = sc.random_configs(60000, 5)
    h = csd.plant_handle(sc.plant)
    h.set_culling(True)
    on = csd.CheckCollisionFreeCuda(q.T, sc.plant)
    h.set_culling(False)
    off = csd.CheckCollisionFreeCuda(q.T, sc.plant)
    h.set_culling(True)
    np.testing.assert_array_equal(on, off)
    assert 0.02 < on.mean() < 0.98  # both verdicts occur
    a = sc.random_configs(3000, 6)
    b = np.clip(a + np.random.default_rng(7).normal(0, 0.3, a.shape), sc.lower(), sc.upper()).astype(np.float32)
    e_on = csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant)
    h.set_culling(False)
    e_off = csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant)
    h.set_culling(True)
    np.testing.assert_array_equal(e_on, e_off)


def test_tree_link_transforms():
    """KinematicTree.compute_link_frame_to_world_transforms (GPU FK) equals the
    batched FK and the oracle's FP64 FK."""
    import os
    from csdecomp_b200.plant import URDFParser
    d = os.path.join(os.path.dirname(__file__), "golden", "loader")
    p = URDFParser()
    p.register_package("loader_assets", d)
    p.parse_directives(os.path.join(d, "cell.yml"))
    kt = p.get_kinematic_tree()
    q = np.array([0.3, -0.7, 0.02], np.float32)
    tfs = kt.compute_link_frame_to_world_transforms(q)
    assert len(tfs) == kt.numLinks()
    batched = csd.ComputeForwardKinematicsCuda(q.reshape(-1, 1), p.get_minimal_plant())[0]
    np.testing.assert_array_equal(np.stack(tfs), batched)
    ref = O.fk(p.get_minimal_plant(), q.reshape(1, -1), fp64=True).reshape(-1, 4, 4).transpose(0, 2, 1)
    np.testing.assert_allclose(np.stack(tfs), ref, atol=1e-5)


def test_staging_wait_gives_up_and_is_reported(plants):
    """The bounded mbarrier wait gives up (nothing completes it), the block
    sets the plant's status word, the host reads and clears it, and the
    context stays usable."""
    import ctypes
    from csdecomp_b200 import _capi as C
    gp = plants["movable_block"]
    h = csd.plant_handle(gp.plant)
    rep = ctypes.c_int32(0)
    assert C.lib().csd_plant_wait_selftest(h.handle, 2000, ctypes.byref(rep)) == C.CSD_OK
    assert rep.value == 1
    t = ctypes.c_int32(1)
    assert C.lib().csd_plant_status(h.handle, ctypes.byref(t), None) == C.CSD_OK and t.value == 0
    rng = np.random.default_rng(4)
    q = (gp.lower + (gp.upper - gp.lower) * rng.random((500, gp.dim))).astype(np.float32)
    band_parity(gp.plant, q)


def edge_band_parity(sc, s, e, mode):
    """GPU edge verdicts against the oracle's (reference rule, early exit): a
    differing edge must hold a point within the contact band; the number of
    points checked equals the oracle's wherever the verdicts agree and the
    edge is free (a colliding edge may stop at another colliding point, since
    the GPU visits points coarse to fine)."""
    gpu, pts = csd.CheckEdgesCollisionFreeCuda(s.T, e.T, sc.plant, 0.01, mode, return_points_checked=True)
    ref, ref_pts = O.check_edges(sc.plant, s, e, 0.01, mode)
    diff = np.nonzero(gpu != ref)[0]
    for i in diff:
        _, sd = O.signed_distance(sc.plant, O.edge_points(s[i], e[i], 0.01, mode))
        assert np.abs(sd).min() <= BAND, i
    free = (gpu == 1) & (ref == 1)
    np.testing.assert_array_equal(pts[free], ref_pts[free])
    return gpu, diff


def test_config2_edges_vs_oracle_full_size():
    """Config 2 as written: 10^5 segments with endpoints uniform in the joint
    limits of the 7-DOF arm (80 spheres + 4 capsules) among 200 world
    primitives, 0.01 rad step, reference (L2) discretisation. Without a
    keep-out nearly every configuration collides, so nearly every segment
    collides at its first point."""
    sc = scenes.edge_check_scene()
    n = 100_000
    s, e = sc.random_configs(n, 201), sc.random_configs(n, 202)
    gpu, diff = edge_band_parity(sc, s, e, csd.CSD_EDGE_L2_REF)
    assert len(diff) <= 3
    assert gpu.sum() <= 10


def test_config2_keepout_edges_vs_oracle():
    """The 0.8 m keep-out variant of config 2 (24% of configurations free),
    10^4 segments with uniform endpoints plus 2,000 short ones, so that free
    edges checked to the end (up to ~660 points each) are part of the case."""
    sc = scenes.edge_check_scene(keepout=0.8)
    rng = np.random.default_rng(203)
    s = sc.random_configs(12_000, 204)
    e = sc.random_configs(12_000, 205)
    e[10_000:] = (s[10_000:] + rng.normal(0, 0.1, (2_000, 7))).astype(np.float32)
    gpu, diff = edge_band_parity(sc, s, e, csd.CSD_EDGE_L2_REF)
    assert len(diff) <= 5
    assert gpu[10_000:].sum() > 50 and gpu.mean() < 0.5
