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
