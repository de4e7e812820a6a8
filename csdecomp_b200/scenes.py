"""Seeded synthetic scenes for the benchmark workloads.

No public dataset is involved: the workloads are random serial revolute arms
with sphere/capsule collision models and axis-aligned world primitives, built
directly as a KinematicTree and then run through the reference's scene rules
(ROBOT/WORLD grouping and pair filter, urdf_parser.cpp:485-616) by
``plant.build_plant``.

Arm: joint i has a fixed transform X_PL_J with translation components drawn
from U[0.05, 0.3] m and a uniformly random rotation, and rotates about its
local z axis within [-pi, pi]. Robot spheres (and capsules) sit along the
segment from a link's origin to the next joint's origin. World primitives sit
on one link welded to the world so that every robot geometry is paired with
every world geometry.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Tuple

import numpy as np

from .plant import (CollisionGeometry, Joint, JointType, KinematicTree, Link, MinimalPlant, SceneInspector,
                    ShapePrimitive, build_plant, make_transform)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform random rotation from a unit quaternion (Shoemake 1992)."""
    u1, u2, u3 = rng.random(3)
    a, b = math.sqrt(1 - u1), math.sqrt(u1)
    x, y, z, w = a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2), \
        b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3)
    R = np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    return R.astype(np.float32)


def _rotation_z_to(v: np.ndarray) -> np.ndarray:
    """A rotation whose third column is v/|v|."""
    z = v / np.linalg.norm(v)
    h = np.array([1.0, 0, 0]) if abs(z[0]) < 0.9 else np.array([0, 1.0, 0])
    x = np.cross(h, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1).astype(np.float32)


@dataclass
class Scene:
    plant: MinimalPlant
    inspector: SceneInspector
    tree: KinematicTree
    seed: int
    description: str

    @property
    def dim(self) -> int:
        return self.plant.kin_tree.num_configuration_variables

    def lower(self) -> np.ndarray:
        return self.tree.getPositionLowerLimits()

    def upper(self) -> np.ndarray:
        return self.tree.getPositionUpperLimits()

    def random_configs(self, n: int, seed: int) -> np.ndarray:
        rng = np.random.default_rng(seed)
        lo, hi = self.lower(), self.upper()
        return (lo + (hi - lo) * rng.random((n, self.dim))).astype(np.float32)


def _add_arm(tree: KinematicTree, geoms: List[CollisionGeometry], rng: np.random.Generator, base_link: int,
             prefix: str, dof: int, num_spheres: int, num_capsules: int) -> None:
    offsets = [rng.uniform(0.05, 0.3, 3) for _ in range(dof + 1)]
    link_ids = []
    parent = base_link
    for i in range(dof):
        li = tree.add_link(Link(name=f"{prefix}link{i + 1}"))
        X = make_transform(random_rotation(rng), offsets[i])
        tree.add_joint(Joint(name=f"{prefix}joint{i + 1}", type=JointType.REVOLUTE, X_PL_J=X,
                             parent_link=parent, child_link=li, axis=np.array([0, 0, 1], np.float32),
                             position_lower_limit=-math.pi, position_upper_limit=math.pi))
        link_ids.append(li)
        parent = li
    # spheres spread evenly over links, along the link segment
    for s in range(num_spheres):
        k = s % dof
        seg = offsets[k + 1]
        c = rng.uniform(0.0, 1.0) * seg + rng.normal(0, 0.01, 3)
        g = CollisionGeometry(type=ShapePrimitive.SPHERE,
                              dimensions=np.array([rng.uniform(0.03, 0.08), -1, -1], np.float32),
                              link_index=link_ids[k], X_L_B=make_transform(np.eye(3), c))
        geoms.append(g)
    for c_i in range(num_capsules):
        k = (c_i * 2 + 1) % dof
        seg = offsets[k + 1]
        r = rng.uniform(0.03, 0.08)
        hl = rng.uniform(0.05, 0.15)
        g = CollisionGeometry(type=ShapePrimitive.CAPSULE, dimensions=np.array([r, 2 * hl, r], np.float32),
                              link_index=link_ids[k],
                              X_L_B=make_transform(_rotation_z_to(seg), 0.5 * seg))
        geoms.append(g)


def _world_primitives(rng: np.random.Generator, obstacle_link: int, num_boxes: int, num_spheres: int,
                      keepout: float, bases: Optional[List[np.ndarray]] = None) -> List[CollisionGeometry]:
    out = []
    bases = bases or [np.zeros(3)]

    def centre(extent: float) -> np.ndarray:
        while True:
            c = rng.uniform(-1.0, 1.0, 3)
            if keepout <= 0 or all(np.linalg.norm(c - b) - extent > keepout for b in bases):
                return c

    for _ in range(num_boxes):
        h = rng.uniform(0.05, 0.3, 3)
        c = centre(float(np.linalg.norm(h)))
        out.append(CollisionGeometry(type=ShapePrimitive.BOX, dimensions=(2 * h).astype(np.float32),
                                     link_index=obstacle_link, X_L_B=make_transform(np.eye(3), c)))
    for _ in range(num_spheres):
        r = rng.uniform(0.05, 0.3)
        c = centre(r)
        out.append(CollisionGeometry(type=ShapePrimitive.SPHERE, dimensions=np.array([r, -1, -1], np.float32),
                                     link_index=obstacle_link, X_L_B=make_transform(np.eye(3), c)))
    return out


def arm_scene(seed: int, num_spheres: int = 40, num_capsules: int = 0, num_world_boxes: int = 20,
              num_world_spheres: int = 0, arms: int = 1, dof_per_arm: int = 7, keepout: float = 0.0,
              description: str = "", arm_spacing: float = 0.6) -> Scene:
    """One (arms=1) or two (arms=2, on a welded base) random revolute arms in a
    field of world primitives. keepout > 0 rejects world primitives within that
    distance of the base."""
    rng = np.random.default_rng(seed)
    tree = KinematicTree()
    tree.add_link(Link(name="world"))
    geoms: List[CollisionGeometry] = []
    if arms == 1:
        _add_arm(tree, geoms, rng, 0, "", dof_per_arm, num_spheres, num_capsules)
    bases = [np.zeros(3)]
    if arms != 1:
        bases = [np.array([0.0, (a - (arms - 1) / 2.0) * arm_spacing, 0.0]) for a in range(arms)]
        base = tree.add_link(Link(name="base"))
        tree.add_joint(Joint(name="base_weld", type=JointType.FIXED, parent_link=0, child_link=base))
        for a in range(arms):
            mount = tree.add_link(Link(name=f"mount{a}"))
            y = (a - (arms - 1) / 2.0) * arm_spacing
            tree.add_joint(Joint(name=f"mount{a}_weld", type=JointType.FIXED, parent_link=base, child_link=mount,
                                 X_PL_J=make_transform(np.eye(3), [0.0, y, 0.0])))
            _add_arm(tree, geoms, rng, mount, f"arm{a}_", dof_per_arm, num_spheres // arms, num_capsules // arms)
    obst = tree.add_link(Link(name="obstacles"))
    tree.add_joint(Joint(name="obstacles_weld", type=JointType.FIXED, parent_link=0, child_link=obst))
    geoms.extend(_world_primitives(rng, obst, num_world_boxes, num_world_spheres, keepout, bases))
    tree.finalize()
    plant, insp = build_plant(tree, geoms)
    return Scene(plant, insp, tree, seed, description)


# --------------------------------------------------------------------------- workloads
POINT_CHECK_SEED = 1000
EDGE_CHECK_SEED = 2000


def point_check_scene(seed: int = POINT_CHECK_SEED) -> Scene:
    """Point-check workload: 7-DOF arm, 40 spheres r~U[0.03,0.08]; 20 world boxes."""
    return arm_scene(seed, num_spheres=40, num_world_boxes=20,
                     description="7-DOF arm, 40 spheres, 20 world boxes")


def edge_check_scene(seed: int = EDGE_CHECK_SEED, keepout: float = 0.0) -> Scene:
    """Edge-check / EI-ZO workload: 7-DOF arm with 80 spheres + 4 capsules;
    200 world primitives (100 boxes, 100 spheres)."""
    return arm_scene(seed, num_spheres=80, num_capsules=4, num_world_boxes=100, num_world_spheres=100,
                     keepout=keepout, description="7-DOF arm, 80 spheres + 4 capsules, 100 boxes + 100 spheres")


BATCH_SEED = 4000


def batch_scene(i: int, seed: int, keepout: float = 0.8) -> Scene:
    """Scene i of the batched-EI-ZO workload: even i a 7-DOF arm (80 spheres + 4
    capsules), odd i a 14-DOF two-arm plant (bases 1.4 m apart, 2 x (40
    spheres + 2 capsules)); U{50..400} world primitives (half boxes, half
    spheres) placed as in edge_check_scene, clear of every arm base."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(50, 401))
    nb = n // 2
    s = int(rng.integers(1 << 30))
    if i % 2 == 0:
        return arm_scene(s, num_spheres=80, num_capsules=4, num_world_boxes=nb, num_world_spheres=n - nb,
                         keepout=keepout, description=f"7-DOF arm, {n} world primitives")
    return arm_scene(s, num_spheres=80, num_capsules=4, num_world_boxes=nb, num_world_spheres=n - nb, arms=2,
                     keepout=keepout, arm_spacing=1.4, description=f"14-DOF two-arm, {n} world primitives")


def batch_scene_cost(i: int, seed: int) -> float:
    """Predicted relative cost of inflating in scene i of the batched workload,
    read from the seed alone (before the scene is built): dimension squared x
    world primitives. The sampler's face loop is dimension-long and the
    regions of the two-arm plant grow several times more faces over more
    iterations; every check visits the world pairs."""
    n = int(np.random.default_rng(seed).integers(50, 401))  # the first draw of batch_scene
    d = 7 if i % 2 == 0 else 14
    return float(d * d * n)


def batch_scene_seeds(count: int, seed: int = BATCH_SEED) -> List[int]:
    rng = np.random.default_rng(seed)
    return [int(rng.integers(1 << 30)) for _ in range(count)]


def batch_scenes(count: int = 256, seed: int = BATCH_SEED, keepout: float = 0.8) -> List[Scene]:
    """`count` scenes for the batched-EI-ZO workload (see batch_scene)."""
    return [batch_scene(i, s, keepout) for i, s in enumerate(batch_scene_seeds(count, seed))]


def seed_edges(scene: Scene, count: int, seed: int, check_points: Callable, check_edges: Callable,
               length: Tuple[float, float] = (0.05, 1.0), draws: int = 8, per_draw: int = 4096) -> list:
    """Up to `count` free seed edges: a free q0 (uniform in the joint limits),
    a direction uniform on the sphere and a length U[length]; kept iff q1 lies
    strictly inside the limits and the edge is collision free. check_points(Q
    [n, d]) -> uint8 [n] and check_edges(Q0, Q1) -> bool [n] are the checkers.
    Returns fewer than `count` edges only when `draws` batches of `per_draw`
    configurations did not yield enough."""
    rng = np.random.default_rng(seed)
    lo, hi = scene.lower(), scene.upper()
    out: list = []
    for _ in range(draws):
        q = scene.random_configs(per_draw, int(rng.integers(1 << 30)))
        free = q[np.asarray(check_points(q)) == 1]
        if len(free) == 0:
            continue
        d = rng.normal(size=free.shape)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        q1 = (free + rng.uniform(length[0], length[1], len(free))[:, None] * d).astype(np.float32)
        inside = np.all((q1 > lo) & (q1 < hi), axis=1)
        a, b = np.ascontiguousarray(free[inside]), np.ascontiguousarray(q1[inside])
        if len(a) == 0:
            continue
        ok = np.asarray(check_edges(a, b)).astype(bool)
        for j in np.nonzero(ok)[0]:
            out.append((a[j].copy(), b[j].copy()))
            if len(out) == count:
                return out
    return out
