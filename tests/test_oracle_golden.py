"""The CPU oracle against the reference's own known-answer tests (no GPU)."""
import numpy as np
import pytest

from oracle import oracle as O


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(O.philox([0xffffffff] * 4, [0xffffffff] * 2)) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0])) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_gaussian_stream_moments():
    z = np.concatenate([O.rng_direction(7, c, 0, s, 14)[:14] for c in range(200) for s in range(20)])
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1.0) < 0.02
    assert abs((z ** 4).mean() - 3.0) < 0.15


@pytest.mark.parametrize("idx", range(4))
def test_fk_golden(plants, golden, idx):
    g = golden["fk"][idx]
    gp = plants[g["plant"]]
    tf32 = O.fk(gp.plant, np.array(g["q"], np.float32))[0]
    tf64 = O.fk(gp.plant, np.array(g["q"], np.float32), fp64=True)[0]
    l = gp.link(g["link"])
    X = np.array(g["X"])
    np.testing.assert_allclose(tf32[l].reshape(4, 4).T, X, atol=2e-6)
    np.testing.assert_allclose(tf64[l].reshape(4, 4).T, X, atol=2e-6)


@pytest.mark.parametrize("rule", [O.RULE_CPU, O.RULE_GPU])
def test_verdict_golden(plants, golden, rule):
    for case in golden["verdicts"]:
        p = plants[case["plant"]].plant
        assert O.check_points(p, np.array(case["free"], np.float32), rule).all(), case["src"]
        assert not O.check_points(p, np.array(case["col"], np.float32), rule).any(), case["src"]


def voxel_grid(case):
    nx, ny, nz = case["grid"]
    sx, sy, sz = case["spacing"]
    off = np.array([-(nx - 1) * sx / 2, -(ny - 1) * sy / 2, 0], np.float32)
    pts = [np.array([ix * sx, iy * sy, iz * sz], np.float32) + off
           for ix in range(nx) for iy in range(ny) for iz in range(nz)]
    return np.array(pts, np.float32)


@pytest.mark.parametrize("rule", [O.RULE_CPU, O.RULE_GPU])
def test_voxel_verdict_golden(plants, golden, rule):
    case = golden["voxel_verdicts"]
    gp = plants[case["plant"]]
    vox = voxel_grid(case)
    f = O.check_points(gp.plant, np.array(case["free"], np.float32), rule, vox, case["radius"], gp.robot_geometry_ids)
    c = O.check_points(gp.plant, np.array(case["col"], np.float32), rule, vox, case["radius"], gp.robot_geometry_ids)
    assert f.all() and not c.any()


def test_visibility_graph_golden(plants, golden):
    case = golden["visibility_graph"]
    gp = plants[case["plant"]]
    nodes = np.array(case["nodes"], np.float32)
    n = len(nodes)
    s, e = zip(*[(nodes[i], nodes[j]) for i in range(n - 1) for j in range(i + 1, n)])
    for mode in (O.EDGE_VG, O.EDGE_L2_REF, O.EDGE_LINF):
        v, _ = O.check_edges(gp.plant, np.array(s), np.array(e), case["step"], mode)
        assert list(v) == case["adjacency_upper"], mode


def test_fp64_agrees_outside_band(plants):
    gp = plants["kinova_on_table"]
    rng = np.random.default_rng(3)
    q = (gp.lower + (gp.upper - gp.lower) * rng.random((2000, gp.dim))).astype(np.float32)
    v = O.check_points(gp.plant, q)
    v64, sd = O.signed_distance(gp.plant, q)
    out = np.abs(sd) > 1e-5
    assert (v[out] == v64[out]).all()
    assert 0.05 < v.mean() < 0.95


def test_edge_rules():
    q1 = np.zeros(7, np.float32)
    q2 = np.full(7, 0.1, np.float32)
    # L2 rule: T = ceil(|dq|/step), end excluded (collision_checker.cpp:44-46)
    assert O.edge_num_points(q1, q2, 0.01, O.EDGE_L2_REF) == int(np.ceil(np.float32(np.sqrt(np.float32(0.07))) / 0.01))
    # Linf rule includes both ends
    assert O.edge_num_points(q1, q2, 0.01, O.EDGE_LINF) == 11
    pts = O.edge_points(q1, q2, 0.01, O.EDGE_LINF)
    np.testing.assert_array_equal(pts[0], q1)
    np.testing.assert_allclose(pts[-1], q2, atol=1e-7)
    # zero-length edge: the reference rule checks no point
    assert O.edge_num_points(q1, q1, 0.01, O.EDGE_L2_REF) == 0


def test_hit_and_run_inside_box():
    d = 7
    A = np.vstack([-np.eye(d), np.eye(d)]).astype(np.float32)
    b = np.concatenate([np.full(d, np.pi), np.full(d, np.pi)]).astype(np.float32)
    s, nf = O.hit_and_run(A, b, np.zeros(d, np.float32), 4000, 50, seed=11)
    assert nf == 0
    assert (A @ s.T <= b[:, None] + 1e-5).all()
    # uniform on [-pi, pi]^7: mean 0, variance pi^2/3
    assert np.abs(s.mean(0)).max() < 0.12
    assert np.abs(s.var(0) - np.pi ** 2 / 3).max() < 0.35


def test_num_samples_unadaptive():
    # M_0 of the EI-ZO defaults (delta_0 = 6 delta / pi^2)
    assert O.num_samples_unadaptive(0.01, np.float32(6 * 0.05 / np.pi ** 2), 0.5) == 2795
    assert O.num_samples_unadaptive(0.01, 0.05, 0.5) == 2397
