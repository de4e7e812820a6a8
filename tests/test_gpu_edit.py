"""EditRegionsCuda on the GPU through the C ABI: the reference's own test
(cuda_edit_regions_test.cpp:79-227), bit-exact replay against the oracle
(the oracle's region editing driven by the GPU's verdicts), ragged inputs and
the reference's error cases."""
import ctypes

import numpy as np
import pytest

import csdecomp_b200 as csd
from csdecomp_b200 import _capi as C
from csdecomp_b200 import scenes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def domain_of(lo, hi):
    d = csd.HPolyhedron()
    d.MakeBox(lo, hi)
    return d


def golden_inputs(plants, golden):
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    col = np.array(g["collisions"], np.float32)
    rep = np.tile(col, (g["repeats"], 1)).T  # dim x 12, as the test's repeated_collisions
    seg = [i for i in range(g["repeats"]) for _ in range(len(col))]
    ls = np.array(g["starts"], np.float32).T
    le = np.array(g["ends"], np.float32).T
    vox = csd.Voxels(np.array(g["voxels"], np.float32).T)
    regions = [domain_of(gp.lower, gp.upper) for _ in range(ls.shape[1])]
    return g, gp, col, rep, seg, ls, le, vox, regions


def gpu_checker(plant, voxels, vr, rids):
    v = csd.Voxels(np.asarray(voxels, np.float32).T) if voxels is not None and len(voxels) else None

    def check(q):
        if v is None:
            return csd.CheckCollisionFreeCuda(q.T, plant)
        return csd.CheckCollisionFreeVoxelsCuda(q.T, v, vr, plant, rids)
    return check


def assert_replay_exact(plant, col, seg, ls, le, regions, rids, vox_rows, vr, opts, out):
    """The oracle's editing with the GPU's verdicts must give the same bits."""
    edited, (proj, opt) = out
    ref_regions, ref_proj, ref_opt = O.edit_regions(
        plant, col.T, seg, ls.T, le.T, [(r.A(), r.b()) for r in regions], rids, vox_rows, vr,
        opts.configuration_margin, opts.bisection_steps, checker=gpu_checker(plant, vox_rows, vr, rids))
    np.testing.assert_array_equal(proj.T, ref_proj)
    np.testing.assert_array_equal(opt.T, ref_opt)
    assert len(edited) == len(ref_regions)
    for e, (A, b) in zip(edited, ref_regions):
        np.testing.assert_array_equal(e.A(), A)
        np.testing.assert_array_equal(e.b(), b)


def test_edit_regions_golden(plants, golden):
    g, gp, col, rep, seg, ls, le, vox, regions = golden_inputs(plants, golden)
    opts = csd.EditRegionsOptions()
    opts.bisection_steps = g["bisection_steps"]
    opts.configuration_margin = g["configuration_margin"]
    edited, (proj, opt) = csd.EditRegionsCuda(rep, seg, ls, le, regions, gp.plant, gp.robot_geometry_ids, vox,
                                              g["voxel_radius"], opts)
    assert proj.shape == opt.shape == rep.shape
    for r, P in enumerate(edited):
        assert P.PointInSet(ls[:, r]) and P.PointInSet(le[:, r])
        for c in range(opt.shape[1]):
            assert not P.PointInSet(opt[:, c])
        for c in range(col.shape[0]):
            assert not P.PointInSet(col[c])
    assert_replay_exact(gp.plant, rep, seg, ls, le, regions, gp.robot_geometry_ids,
                        np.array(g["voxels"], np.float32), g["voxel_radius"], opts, (edited, (proj, opt)))
    # the oracle's own verdicts agree on this scene as well
    ref_regions, ref_proj, ref_opt = O.edit_regions(gp.plant, rep.T, seg, ls.T, le.T,
                                                    [(r.A(), r.b()) for r in regions], gp.robot_geometry_ids,
                                                    g["voxels"], g["voxel_radius"], g["configuration_margin"],
                                                    g["bisection_steps"])
    np.testing.assert_array_equal(opt.T, ref_opt)


def test_edit_regions_unbisected(plants, golden):
    g, gp, col, rep, seg, ls, le, vox, regions = golden_inputs(plants, golden)
    opts = csd.EditRegionsOptions(bisection_steps=g["unbisected_steps"])
    _, (_, opt) = csd.EditRegionsCuda(rep, seg, ls, le, regions, gp.plant, gp.robot_geometry_ids, vox,
                                      g["voxel_radius"], opts)
    c = g["unbisected_col"]
    assert np.linalg.norm(opt[:, c] - col[c]) <= g["unbisected_tol"]


@pytest.mark.parametrize("arms,voxels", [(1, False), (1, True), (2, False)])
def test_edit_regions_arm_replay(arms, voxels):
    """Thousands of collisions over ragged regions (some with none, extra
    faces on others), segment indices shuffled: bit-exact against the replay."""
    sc = scenes.arm_scene(60 + arms, num_spheres=40, num_capsules=2, num_world_boxes=30, num_world_spheres=20,
                          arms=arms, keepout=0.5)
    d = sc.dim
    rng = np.random.default_rng(7 + arms)
    lo, hi = sc.lower(), sc.upper()
    m = 37
    ls = np.zeros((d, m), np.float32)
    le = np.zeros((d, m), np.float32)
    regions, boxes = [], []
    for r in range(m):
        c = (lo + (hi - lo) * rng.uniform(0.3, 0.7, d)).astype(np.float32)
        w = ((hi - lo) * rng.uniform(0.1, 0.3, d)).astype(np.float32)
        blo, bhi = np.maximum(lo, c - w), np.minimum(hi, c + w)
        P = domain_of(blo, bhi)
        ls[:, r] = c - 0.3 * w
        le[:, r] = c + 0.3 * w
        if r % 3 == 1:  # an extra oblique face that keeps the segment
            a = rng.normal(size=d).astype(np.float32)
            a /= np.linalg.norm(a)
            off = np.float32(max(a @ ls[:, r], a @ le[:, r]) + 0.05)
            P = csd.HPolyhedron(np.vstack([P.A(), a]), np.append(P.b(), off))
        regions.append(P)
        boxes.append((blo, bhi))
    rids = sc.inspector.robot_geometry_ids
    vox_rows = rng.uniform(-0.8, 0.8, (300, 3)).astype(np.float32) if voxels else None
    vr = 0.03
    chk = gpu_checker(sc.plant, vox_rows, vr, rids)
    cols, segs = [], []
    for r in range(m):
        if r % 5 == 4:  # no collisions: these regions come back unchanged
            continue
        blo, bhi = boxes[r]
        q = (blo + (bhi - blo) * rng.random((200, d))).astype(np.float32)
        q = q[chk(q) == 0]
        cols.append(q)
        segs.append(np.full(q.shape[0], r))
    q = sc.random_configs(2000, 11 + arms)  # collisions anywhere, mostly outside their region
    q = q[chk(q) == 0]
    cols.append(q)
    segs.append(rng.choice([r for r in range(m) if r % 5 != 4], q.shape[0]))
    col = np.concatenate(cols)
    seg = np.concatenate(segs)
    perm = rng.permutation(col.shape[0])
    col, seg = col[perm], seg[perm]
    opts = csd.EditRegionsOptions()
    out = csd.EditRegionsCuda(col.T, seg, ls, le, regions, sc.plant, rids,
                              csd.Voxels(vox_rows.T) if voxels else csd.Voxels(), vr, opts)
    edited = out[0]
    for r in range(m):
        assert edited[r].PointInSet(ls[:, r]) and edited[r].PointInSet(le[:, r])
        if not (seg == r).any():
            assert edited[r] is regions[r]
    assert sum(e.b().size - r.b().size for e, r in zip(edited, regions)) > m
    assert_replay_exact(sc.plant, col.T, seg, ls, le, regions, rids, vox_rows, vr, opts, out)


def test_edit_regions_errors(plants, golden):
    g, gp, col, rep, seg, ls, le, vox, regions = golden_inputs(plants, golden)
    opts = csd.EditRegionsOptions()
    vr = g["voxel_radius"]
    rids = gp.robot_geometry_ids
    bad_ls = ls.copy()
    bad_ls[:, 1] = [2.5, 0.0]  # outside the domain box
    with pytest.raises(RuntimeError, match="line start is not contained in region 1"):
        csd.EditRegionsCuda(rep, seg, bad_ls, le, regions, gp.plant, rids, vox, vr, opts)
    with pytest.raises(RuntimeError, match="No collisions"):
        csd.EditRegionsCuda(np.zeros((2, 0), np.float32), [], ls, le, regions, gp.plant, rids, vox, vr, opts)
    with pytest.raises(IndexError):
        csd.EditRegionsCuda(rep, [5] * rep.shape[1], ls, le, regions, gp.plant, rids, vox, vr, opts)
    with pytest.raises(ValueError):
        csd.EditRegionsCuda(rep, seg, ls, le, regions, gp.plant, rids, vox, 0.0, opts)
    with pytest.raises(ValueError):
        csd.EditRegionsCuda(rep, seg, ls, le, regions, gp.plant, [], vox, vr, opts)
    with pytest.raises(ValueError):
        csd.EditRegionsCuda(rep, seg, ls[:, :2], le[:, :2], regions, gp.plant, rids, vox, vr, opts)
    with pytest.raises(RuntimeError, match="Voxel buffer"):
        csd.EditRegionsCuda(rep, seg, ls, le, regions, gp.plant, rids, csd.Voxels(np.zeros((3, 10001))), vr, opts)
    # the C ABI refuses an out-of-range segment index by itself
    h = csd.plant_handle(gp.plant)
    q = np.ascontiguousarray(rep.T)
    s = np.full(q.shape[0], 3, np.uint32)
    A = np.ascontiguousarray(np.concatenate([r.A() for r in regions]), np.float32)
    b = np.ascontiguousarray(np.concatenate([r.b() for r in regions]), np.float32)
    off = np.array([0, 4, 8, 12], np.int32)
    ids = np.array(rids, np.int32)
    out = [np.zeros((12 + q.shape[0], 2), np.float32), np.zeros(12 + q.shape[0], np.float32), np.zeros(3, np.int32),
           np.zeros_like(q), np.zeros_like(q)]
    o = opts._c()
    rc = C.lib().csd_edit_regions(h.handle, C.ptr(q), C.ptr(s), ctypes.c_int64(q.shape[0]),
                                  C.ptr(np.ascontiguousarray(ls.T)), C.ptr(np.ascontiguousarray(le.T)), 3, C.ptr(A),
                                  C.ptr(b), C.ptr(off), None, 0, ctypes.c_float(vr), C.ptr(ids), ids.size,
                                  ctypes.byref(o), *[C.ptr(x) for x in out])
    assert rc == C.CSD_ERR_INVALID


def test_edit_regions_collision_on_segment(plants, golden):
    """A collision lying on its own segment gives a zero normal (left
    unnormalised, as Eigen's normalize leaves a zero vector) and a face
    0 . x <= 2e-6 that every point satisfies."""
    g = golden["edit_regions_2d"]
    gp = plants[g["plant"]]
    regions = [domain_of(gp.lower, gp.upper)]
    ls = np.array([[0.5], [0.5]], np.float32)
    le = np.array([[1.5], [1.5]], np.float32)
    col = np.array([[1.0], [1.0]], np.float32)  # inside the top-right box, on the segment
    opts = csd.EditRegionsOptions()
    edited, (proj, opt) = csd.EditRegionsCuda(col, [0], ls, le, regions, gp.plant, gp.robot_geometry_ids,
                                              csd.Voxels(), 0.05, opts)
    np.testing.assert_array_equal(proj, col)
    np.testing.assert_array_equal(opt, col)
    A, b = edited[0].A(), edited[0].b()
    assert A.shape[0] == 5
    np.testing.assert_array_equal(A[4], [0, 0])
    assert 0 < b[4] < 1e-5
    ref, _, _ = O.edit_regions(gp.plant, col.T, [0], ls.T, le.T, [(regions[0].A(), regions[0].b())],
                               gp.robot_geometry_ids)
    np.testing.assert_array_equal(A, ref[0][0])
    np.testing.assert_array_equal(b, ref[0][1])
