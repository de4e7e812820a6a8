"""The batched EI-ZO (the benchmark's own path) against the oracle, slot by
slot, at the benchmark's options: 2,000 particles, 50 mixing steps, 9
bisection steps, run to admissibility.

The oracle's EI-ZO (restating executeEizo,
csdecomp/src/planning/cuda_edge_inflation_zero_order.cu:109-338 and
cuda_set_builder_utils.cu:25-455) is driven by the GPU checker's verdicts on
the slot's plant; sampling, compaction, projection, bisection, distances,
argmin, face placement and redundancy marking are then the oracle's own, so a
slot whose region (A, b) and iteration count equal the replay's is pinned to
the oracle end to end. Scenes and seed edges are the benchmark workload's
first two (scene 0: 7-DOF arm; scene 1: 14-DOF two-arm plant).
"""
import numpy as np
import pytest

import bench
import csdecomp_b200 as csd
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_checkers(sc):
    return (lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
            lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant))


@pytest.fixture(scope="module")
def bench_slots():
    seeds, _, n = bench.scene_ranges(1)
    items, skipped = bench.workload(0, 2, 1, gpu_checkers, seeds, n)
    assert skipped == 0
    assert [sc.dim for sc, _ in items] == [7, 14]
    return items


def replay(sc, q0, q1, opt, capacity):
    A0, b0 = bench.box_domain(sc)
    return O.eizo(sc.plant, q0, q1, A0, b0, opt, sc.inspector.robot_geometry_ids, capacity=capacity,
                  checker=lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant))


@pytest.fixture(scope="module")
def oracle_regions(bench_slots):
    opt = csd.EizoOptions(**bench.EIZO_KW)
    return [replay(sc, e[0][0], e[0][1], opt, bench.FACE_CAPACITY) for sc, e in bench_slots]


def run_batch(bench_slots, variant):
    scs = [sc for sc, _ in bench_slots]
    opt = csd.EizoOptions(**bench.EIZO_KW)
    batch = csd.BatchedEdgeInflator([sc.plant for sc in scs], opt, max_slots=len(scs),
                                    face_capacity=bench.FACE_CAPACITY,
                                    autotune_iterations=4 if variant is None else 0)
    if variant is not None:
        batch.set_shapes(variant, 128)
    doms = []
    for sc in scs:
        d = csd.HPolyhedron()
        d.MakeBox(sc.lower(), sc.upper())
        doms.append(d)
    got = batch.inflate(list(range(len(scs))), [e[0][0] for _, e in bench_slots], [e[0][1] for _, e in bench_slots],
                        doms)
    return got, batch


VARIANTS = {name: i for i, name in enumerate(csd.BatchedEdgeInflator.SAMPLE_VARIANTS)}


@pytest.mark.parametrize("variant", [None] + sorted(set(VARIANTS.values())))
def test_batch_slots_equal_oracle_replay(bench_slots, oracle_regions, variant):
    """Every sampler variant (and the autotuned choice the benchmark makes)
    reproduces the oracle's regions bit for bit on a 7-DOF and a 14-DOF slot."""
    got, batch = run_batch(bench_slots, variant)
    for i, (P, (A, b, iters)) in enumerate(zip(got, oracle_regions)):
        np.testing.assert_array_equal(P.A(), A, err_msg=f"slot {i} (dim {bench_slots[i][0].dim})")
        np.testing.assert_array_equal(P.b(), b, err_msg=f"slot {i}")
        assert int(batch.last_iterations[i]) == len(iters), f"slot {i}"
    # the regions grew past the domain box (the replay is not vacuous)
    assert got[0].A().shape[0] > 14 + 10 and got[1].A().shape[0] > 28 + 10


def test_oracle_replay_iterations_are_consistent(oracle_regions):
    """Per-iteration bookkeeping of the replay: faces placed add up to the
    region, and every iteration but the last failed the unadaptive test."""
    for (A, b, iters), dom_faces in zip(oracle_regions, (14, 28)):
        assert A.shape[0] == dom_faces + sum(r["num_faces_placed"] for r in iters)
        assert all(r["num_collisions_unadaptive"] > r["collisions_threshold"] for r in iters[:-1])
        assert iters[-1]["num_collisions_unadaptive"] <= iters[-1]["collisions_threshold"]
