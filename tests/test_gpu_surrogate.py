"""Surrogate-guided batched EI-ZO: the trained bank orders the checks, the
exact checker judges every verdict. Regions stay valid (contain the seed
segment, pass the admissibility spot check) and fewer configurations are
checked than without the surrogate."""
import numpy as np
import pytest

import csdecomp_b200 as csd
from csdecomp_b200 import scenes
from csdecomp_b200.surrogate import CollisionSurrogate, training_set

pytestmark = pytest.mark.gpu


def setup_module(_):
    global S7, S14, EDGES, DOMS
    S7 = scenes.arm_scene(41, num_spheres=40, num_capsules=2, num_world_boxes=40, num_world_spheres=40, keepout=0.8)
    S14 = scenes.arm_scene(42, num_spheres=40, num_capsules=2, num_world_boxes=30, num_world_spheres=30, arms=2,
                           keepout=0.9, arm_spacing=1.4)
    EDGES = []
    for i, sc in enumerate((S7, S14)):
        e = scenes.seed_edges(sc, 3, 50 + i, lambda q, sc=sc: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                              lambda a, b, sc=sc: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant),
                              length=(0.2, 0.6))
        assert len(e) == 3
        EDGES.append(e)
    DOMS = []
    for sc in (S7, S14):
        d = csd.HPolyhedron()
        d.MakeBox(sc.lower(), sc.upper())
        DOMS.append(d)


def trained_bank(epochs=6):
    bank = CollisionSurrogate([S7.dim, S14.dim], seed=7)
    xs, ys = [], []
    for i, sc in enumerate((S7, S14)):
        x, y = training_set(sc, EDGES[i], 16384, seed=100 + i)
        xs.append(x)
        ys.append(y)
    hist = bank.train(xs, ys, batch=512, epochs=epochs, lr=2e-3)
    return bank, hist, ys


def run(bank, opt):
    b = csd.BatchedEdgeInflator([S7.plant, S14.plant], opt, max_slots=6, face_capacity=400)
    if bank is not None:
        b.set_surrogate(bank, 0.1)
    slots = [0, 1, 0, 1, 0, 1]
    starts = [EDGES[p][k // 2][0] for k, p in enumerate(slots)]
    ends = [EDGES[p][k // 2][1] for k, p in enumerate(slots)]
    regs = b.inflate(slots, starts, ends, [DOMS[p] for p in slots])
    return regs, b.last_configs_checked.copy(), slots, starts, ends


def contains_segment(P, a, b):
    for t in np.linspace(0, 1, 11):
        q = a + t * (b - a)
        if not np.all(P.A() @ q <= P.b() + 1e-5):
            return False
    return True


def test_surrogate_batch_checks_fewer_configurations_and_keeps_regions_valid():
    bank, hist, ys = trained_bank()
    assert hist[-10:].mean() < hist[:10].mean()
    opt = csd.EizoOptions(num_particles=600, mixing_steps=20, max_iterations=40)
    plain, cfg_plain, slots, starts, ends = run(None, opt)
    surr, cfg_surr, _, _, _ = run(bank, opt)
    for P, p, a, b in zip(surr, slots, starts, ends):
        assert contains_segment(P, a, b)
        # admissibility spot check: uniform samples of the region rarely collide
        sc = (S7, S14)[p]
        smp = csd.UniformSampleInHPolyhedraCuda([P], a, 2000, 30, 11)[0]
        free = csd.CheckCollisionFreeCuda(smp, sc.plant)
        assert (free == 0).mean() < 0.05
    assert cfg_surr.sum() < 0.9 * cfg_plain.sum(), (cfg_surr.sum(), cfg_plain.sum())


def test_untrained_surrogate_still_gives_valid_regions():
    bank = CollisionSurrogate([S7.dim, S14.dim], seed=3)
    opt = csd.EizoOptions(num_particles=600, mixing_steps=20, max_iterations=40)
    surr, _, slots, starts, ends = run(bank, opt)
    for P, a, b in zip(surr, starts, ends):
        assert contains_segment(P, a, b)


def test_surrogate_must_match_the_plants():
    b = csd.BatchedEdgeInflator([S7.plant, S14.plant], csd.EizoOptions(num_particles=100, max_iterations=5), 2, 100)
    with pytest.raises(ValueError):
        b.set_surrogate(CollisionSurrogate([S7.dim]), 0.1)
    with pytest.raises(RuntimeError):
        b.set_surrogate(CollisionSurrogate([S14.dim, S7.dim]), 0.1)


def edge_set(sc, n, seed):
    """Edges from free starts, mixed verdicts: lengths U[0.05, 1.0] rad."""
    rng = np.random.default_rng(seed)
    q = sc.random_configs(8 * n, seed)
    q0 = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1][:n]
    d = rng.normal(size=q0.shape)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q1 = np.clip(q0 + rng.uniform(0.05, 1.0, (len(q0), 1)) * d, sc.lower(), sc.upper()).astype(np.float32)
    return q0, q1


@pytest.mark.parametrize("mode", [csd.CSD_EDGE_L2_REF, csd.CSD_EDGE_LINF, csd.CSD_EDGE_VG])
def test_ranked_edges_exact(mode):
    """Ranking only reorders: verdicts equal the unranked check for an
    untrained net, a trained one and every candidate count."""
    bank, _, _ = trained_bank(epochs=2)
    raw = CollisionSurrogate([S7.dim, S14.dim], seed=3)
    for net, sc in enumerate((S7, S14)):
        q0, q1 = edge_set(sc, 400, 11 + net)
        ref, ref_pts = csd.CheckEdgesCollisionFreeCuda(q0.T, q1.T, sc.plant, 0.01, mode, return_points_checked=True)
        assert 0 < ref.mean() < 1
        for b in (bank, raw):
            for top in (0, 1, 8, 32):
                got, pts = csd.CheckEdgesCollisionFreeRankedCuda(q0.T, q1.T, sc.plant, b, net, 0.01, mode, top,
                                                                 return_points_checked=True)
                np.testing.assert_array_equal(got, ref)
                # free edges: every point is checked exactly once
                np.testing.assert_array_equal(pts[ref == 1], ref_pts[ref == 1])
                if top == 0:
                    np.testing.assert_array_equal(pts, ref_pts)


def test_ranked_edges_exit_earlier():
    """A trained net moves colliding edges' first hit earlier."""
    bank, _, _ = trained_bank()
    for net, sc in enumerate((S7, S14)):
        q0, q1 = edge_set(sc, 600, 31 + net)
        ref, ref_pts = csd.CheckEdgesCollisionFreeCuda(q0.T, q1.T, sc.plant, 0.01, return_points_checked=True)
        got, pts = csd.CheckEdgesCollisionFreeRankedCuda(q0.T, q1.T, sc.plant, bank, net, 0.01, top=8,
                                                         return_points_checked=True)
        np.testing.assert_array_equal(got, ref)
        col = ref == 0
        assert col.sum() > 50
        assert pts[col].mean() < ref_pts[col].mean(), (pts[col].mean(), ref_pts[col].mean())


def test_ranked_edges_bad_arguments():
    bank, _, _ = trained_bank(epochs=1)
    q0, q1 = edge_set(S7, 8, 5)
    with pytest.raises(csd.CsdError):
        csd.CheckEdgesCollisionFreeRankedCuda(q0.T, q1.T, S7.plant, bank, 1)  # the 14-D net on the 7-D plant
    with pytest.raises(ValueError):
        csd.CheckEdgesCollisionFreeRankedCuda(q0.T, q1.T, S7.plant, bank, 0, top=33)
    with pytest.raises(ValueError):
        csd.CheckEdgesCollisionFreeRankedCuda(q0.T, q1.T, S7.plant, bank, 5)


def test_surrogate_turns_itself_off_where_ordering_cannot_save():
    """With num_particles = N_0 = 4000 and stop probability ~0, the first
    iteration of a slot checks every sample (it cannot hold num_particles
    collisions before its last sample), so ordering saves nothing: each slot
    checks in sample order from its second iteration on and the call
    continues with the batched form's graph (6 kernels per iteration instead
    of 13). The regions equal the batched form's: no colliding sample was
    left unchecked."""
    bank, _, _ = trained_bank(epochs=2)
    opt = csd.EizoOptions(num_particles=4000, mixing_steps=20, max_iterations=12)
    plain, cfg_plain, slots, starts, ends = run(None, opt)
    b = csd.BatchedEdgeInflator([S7.plant, S14.plant], opt, max_slots=6, face_capacity=400, autotune_iterations=0)
    b.set_surrogate(bank, 1e-30)  # a slot that is decided inadmissible never stops early
    surr = b.inflate(slots, starts, ends, [DOMS[p] for p in slots])
    for P, R in zip(surr, plain):
        np.testing.assert_array_equal(P.A(), R.A())
        np.testing.assert_array_equal(P.b(), R.b())
    np.testing.assert_array_equal(b.last_configs_checked, cfg_plain)
    iters = int(b.last_iterations.max())
    assert iters >= 2
    # init kernel + one surrogate iteration (sample, score, sort, 3 x (check, tally), compaction,
    # bisect, faces, step) + batched iterations (sample, check, compaction, bisect, faces, step)
    assert b.last_kernel_launches == 1 + 13 + 6 * (iters - 1)
