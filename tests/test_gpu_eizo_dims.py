"""EI-ZO at every dimension class of the sampler's draw layout: the single
inflation and the batched form against the oracle's replay, bit for bit.

The sampler draws a whole Philox block per slot (two Gaussian pairs, or a
pair and the theta uniform), so the layout changes with ceil(dim/2): the
number of blocks per step, whether the theta uniform opens or closes its
block, how many steps a group of 8 lanes draws at once, and the 8 / 16
coordinate split of the face rows. These arms span dims 1 to 16 through each
of those cases; the oracle (restating executeEizo,
csdecomp/src/planning/cuda_edge_inflation_zero_order.cu:109-338, with the
GPU checker's verdicts) decides every sample, face and iteration count.
"""
import numpy as np
import pytest

import csdecomp_b200 as csd
from csdecomp_b200 import scenes
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OPT = dict(num_particles=300, mixing_steps=12, bisection_steps=9, max_hyperplanes_per_iteration=10,
           epsilon=0.01, delta=0.05, tau=0.5, max_iterations=4, configuration_margin=0.01, seed=77)
CAP = 200


def arm(d):
    return scenes.arm_scene(500 + d, num_spheres=max(8, 2 * d), num_world_boxes=12, num_world_spheres=12,
                            dof_per_arm=d, keepout=0.6)


def box(sc):
    p = csd.HPolyhedron()
    p.MakeBox(sc.lower(), sc.upper())
    return p


@pytest.mark.parametrize("d", [1, 2, 3, 5, 6, 8, 9, 11, 12, 15, 16])
def test_single_and_batched_equal_oracle_replay(d):
    sc = arm(d)
    cp = lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant)  # noqa: E731
    ce = lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant)  # noqa: E731
    edges = scenes.seed_edges(sc, 1, 900 + d, cp, ce)
    assert edges, f"no free seed edge at dim {d}"
    q0, q1 = edges[0]
    opt = csd.EizoOptions(**OPT)
    dom = box(sc)
    A, b, iters = O.eizo(sc.plant, q0, q1, dom.A(), dom.b(), opt, sc.inspector.robot_geometry_ids, capacity=CAP,
                         checker=cp)
    inf = csd.CudaEdgeInflator(sc.plant, sc.inspector.robot_geometry_ids, opt, dom, face_capacity=CAP)
    single = inf.inflateEdge(q0, q1, None, 0.0, verbose=False)
    np.testing.assert_array_equal(single.A(), A, err_msg=f"single, dim {d}")
    np.testing.assert_array_equal(single.b(), b, err_msg=f"single, dim {d}")
    batch = csd.BatchedEdgeInflator([sc.plant], opt, max_slots=1, face_capacity=CAP, autotune_iterations=0)
    got = batch.inflate([0], [q0], [q1], [dom])[0]
    np.testing.assert_array_equal(got.A(), A, err_msg=f"batched, dim {d}")
    np.testing.assert_array_equal(got.b(), b, err_msg=f"batched, dim {d}")
    assert int(batch.last_iterations[0]) == len(iters)
    if d > 1:  # faces were placed: the replay compares sampled regions, not just the box (the 1-DOF arm's
        # segment is admissible at once; its samples and checks are still the oracle's)
        assert A.shape[0] > 2 * d
