"""Plant model: kinematic tree, collision geometries, collision pairs.

Host-side mirror of the reference's model types and of the parts of its URDF
parser that decide what the hot path computes:

* ``MinimalKinematicTree`` / ``MinimalPlant``  -- csdecomp/src/plant/minimal_kinematic_tree.h:18-53,
  csdecomp/src/plant/minimal_plant.h:16-39 (stored here as numpy tables, no fixed capacities);
* ``KinematicTree.finalize``                    -- csdecomp/src/plant/kinematic_tree.cpp:82-146
  (joint -> configuration index, DFS traversal order with an explicit stack);
* ``URDFParser``                                -- csdecomp/src/plant/urdf_parser.cpp:78-200, 208-466
  (links first, then joints; ``origin`` rpy -> Rz*Ry*Rx; box dimensions are full extents;
  sphere dimensions are (r, -1, -1)), directives :618-778;
* ``URDFParser.finalize_scene``                 -- csdecomp/src/plant/urdf_parser.cpp:485-616
  (ROBOT/WORLD grouping through fixed joints and the collision-pair filter).

Capsules are accepted (dimensions (r, length, r), axis = local z); the
reference parser rejects them (urdf_parser.cpp:450-452).
"""
from __future__ import annotations

import enum
import math
import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

FLT_MAX = float(np.finfo(np.float32).max)


class JointType(enum.IntEnum):
    FIXED = 0
    REVOLUTE = 1
    PRISMATIC = 2


class ShapePrimitive(enum.IntEnum):
    BOX = 0
    SPHERE = 1
    CYLINDER = 2
    CAPSULE = 3


class CollisionGroup(enum.IntEnum):
    ROBOT = 0
    WORLD = 1
    VOXELS = 2


def _f32(x) -> np.float32:
    return np.float32(x)


def _mat3(a, b):
    """3x3 product in FP64, each entry summed k = 0, 1, 2 (the native loader's order)."""
    out = [[0.0] * 3 for _ in range(3)]
    for i in range(3):
        for j in range(3):
            s = 0.0
            for k in range(3):
                s += a[i][k] * b[k][j]
            out[i][j] = s
    return out


def rpy_to_matrix(r: float, p: float, y: float) -> np.ndarray:
    """(Rz(y) * Ry(p)) * Rx(r) (urdf_parser.cpp:370-375), evaluated in FP64, stored FP32."""
    cr, sr = math.cos(r), math.sin(r)
    cp, sp = math.cos(p), math.sin(p)
    cy, sy = math.cos(y), math.sin(y)
    rx = [[1.0, 0.0, 0.0], [0.0, cr, -sr], [0.0, sr, cr]]
    ry = [[cp, 0.0, sp], [0.0, 1.0, 0.0], [-sp, 0.0, cp]]
    rz = [[cy, -sy, 0.0], [sy, cy, 0.0], [0.0, 0.0, 1.0]]
    return np.array(_mat3(_mat3(rz, ry), rx), np.float64).astype(np.float32)


def unit_axis(a) -> np.ndarray:
    """a / |a| in FP32 with |a|^2 summed x, y, z (Eigen's normalized() on a Vector3f)."""
    x, y, z = (np.float32(v) for v in a)
    n = np.float32(np.sqrt(np.float32(np.float32(np.float32(x * x) + np.float32(y * y)) + np.float32(z * z))))
    return np.array([x / n, y / n, z / n], np.float32)


def make_transform(R: np.ndarray, t: Sequence[float]) -> np.ndarray:
    X = np.eye(4, dtype=np.float32)
    X[:3, :3] = R
    X[:3, 3] = np.asarray(t, dtype=np.float32)
    return X


@dataclass
class CollisionGeometry:
    type: int = ShapePrimitive.BOX
    dimensions: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    link_index: int = 0
    group: int = CollisionGroup.ROBOT
    X_L_B: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))


@dataclass
class Joint:
    name: str = ""
    type: int = JointType.FIXED
    X_PL_J: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))
    parent_link: int = -1
    child_link: int = -1
    axis: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))
    position_lower_limit: float = -FLT_MAX
    position_upper_limit: float = FLT_MAX


@dataclass
class Link:
    name: str = ""
    parent_joint: int = -1
    child_joints: List[int] = field(default_factory=list)


class KinematicTree:
    """Links/joints with the finalize() rules of kinematic_tree.cpp:14-146."""

    def __init__(self):
        self.links: List[Link] = []
        self.joints: List[Joint] = []
        self.link_name_to_index: Dict[str, int] = {}
        self.joint_name_to_index: Dict[str, int] = {}
        self._finalized = False
        self.joint_idx_to_config_idx: List[int] = []
        self.joint_traversal_sequence: List[int] = []
        self.num_configuration_variables = 0
        self.position_lower_limits: List[float] = []
        self.position_upper_limits: List[float] = []

    # kinematic_tree.cpp:14-28
    def add_link(self, link: Link) -> int:
        if link.name in self.link_name_to_index:
            raise RuntimeError(f"Duplicate link name detected in URDF. Name : {link.name}")
        if self._finalized:
            raise RuntimeError("Cannot add link to finalized tree.")
        idx = len(self.links)
        self.links.append(link)
        self.link_name_to_index[link.name] = idx
        return idx

    # kinematic_tree.cpp:30-52
    def add_joint(self, joint: Joint) -> int:
        if joint.name in self.joint_name_to_index:
            raise RuntimeError("Duplicate joint name detected in URDF.")
        if self._finalized:
            raise RuntimeError("Cannot add joint to finalized tree.")
        if joint.parent_link == -1 or joint.child_link == -1:
            raise RuntimeError("Parent or child link not found for joint: " + joint.name)
        idx = len(self.joints)
        self.joints.append(joint)
        self.joint_name_to_index[joint.name] = idx
        self.links[joint.parent_link].child_joints.append(idx)
        self.links[joint.child_link].parent_joint = idx
        return idx

    def get_link_index(self, name: str) -> int:
        if name not in self.link_name_to_index:
            raise RuntimeError(f"[KinematicTree] Invalid link name {name}")
        return self.link_name_to_index[name]

    getLinkIndexByName = get_link_index

    # kinematic_tree.cpp:82-146
    def finalize(self) -> None:
        self._finalized = True
        self.num_configuration_variables = 0
        self.joint_idx_to_config_idx = []
        for j in self.joints:
            if j.type != JointType.FIXED:
                self.joint_idx_to_config_idx.append(self.num_configuration_variables)
                self.num_configuration_variables += 1
            else:
                self.joint_idx_to_config_idx.append(-1)
        # DFS with an explicit stack starting at the root's child joints
        seq: List[int] = []
        stack = list(self.links[0].child_joints)
        while stack:
            j = stack.pop()
            seq.append(j)
            stack.extend(self.links[self.joints[j].child_link].child_joints)
        self.joint_traversal_sequence = seq
        self.position_lower_limits = [j.position_lower_limit for j in self.joints if j.type != JointType.FIXED]
        self.position_upper_limits = [j.position_upper_limit for j in self.joints if j.type != JointType.FIXED]

    def is_finalized(self) -> bool:
        return self._finalized

    isFinalized = is_finalized

    # kinematic_tree.cpp:69-80, 148-165
    def get_link_name(self, index: int) -> str:
        for name, i in self.link_name_to_index.items():
            if i == index:
                return name
        raise RuntimeError("link index not found")

    def get_link(self, index: int) -> Link:
        if not 0 <= index < len(self.links):
            raise IndexError("link index out of range")
        return self.links[index]

    def get_joint_index(self, name: str) -> int:
        return self.joint_name_to_index.get(name, -1)

    def get_joint(self, index: int) -> Joint:
        if not 0 <= index < len(self.joints):
            raise IndexError("joint index out of range")
        return self.joints[index]

    def get_links(self) -> List[Link]:
        return self.links

    def get_joints(self) -> List[Joint]:
        return self.joints

    def get_leaf_link_indices(self) -> List[int]:
        return [i for i, l in enumerate(self.links) if not l.child_joints]

    def compute_link_frame_to_world_transforms(self, joint_values) -> List[np.ndarray]:
        """computeLinkFrameToWorldTransforms (kinematic_tree.cpp:195-240): one
        4 x 4 link-to-world transform per link, evaluated on the GPU."""
        if not self._finalized:
            raise RuntimeError("KinematicTree is not finalized")
        q = np.asarray(joint_values, np.float32).reshape(-1)
        if q.size != self.num_configuration_variables:
            raise ValueError(f"Incorrect number of configuration varialbes added, there are "
                             f"{self.num_configuration_variables} active joints and {q.size} configuration "
                             f"values were provided")
        from .api import ComputeForwardKinematicsCuda
        tf = ComputeForwardKinematicsCuda(q.reshape(-1, 1), self.get_minimal_kinematic_tree())[0]
        return [tf[l].copy() for l in range(tf.shape[0])]

    def numLinks(self) -> int:
        return len(self.links)

    def numJoints(self) -> int:
        return len(self.joints)

    def numConfigurationVariables(self) -> int:
        return self.num_configuration_variables

    def getPositionLowerLimits(self) -> np.ndarray:
        return np.asarray(self.position_lower_limits, dtype=np.float32)

    def getPositionUpperLimits(self) -> np.ndarray:
        return np.asarray(self.position_upper_limits, dtype=np.float32)

    get_position_lower_limits = getPositionLowerLimits
    get_position_upper_limits = getPositionUpperLimits
    num_links = numLinks

    def get_minimal_kinematic_tree(self) -> "MinimalKinematicTree":
        return MinimalKinematicTree.from_tree(self)

    getMyMinimalKinematicTreeStruct = get_minimal_kinematic_tree


@dataclass
class MinimalJoint:
    """minimal_kinematic_tree.h:18-26."""
    type: int = JointType.FIXED
    X_PL_J: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))
    index: int = 0
    parent_link: int = -1
    child_link: int = -1
    axis: np.ndarray = field(default_factory=lambda: np.zeros(3, np.float32))


@dataclass
class MinimalLink:
    """minimal_kinematic_tree.h:31-37 (the child joint array holds exactly the
    link's child joints; the reference pads it to MAX_CHILD_JOINT_COUNT)."""
    index: int = 0
    parent_joint_index: int = -1
    child_joint_index_array: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    num_child_joints: int = 0


@dataclass
class MinimalKinematicTree:
    """Table form of minimal_kinematic_tree.h:42-53 (no fixed capacities);
    ``joints`` and ``links`` give the reference's per-element structs."""

    joint_type: np.ndarray
    joint_X_PL_J: np.ndarray  # [J,4,4]
    joint_parent_link: np.ndarray
    joint_child_link: np.ndarray
    joint_axis: np.ndarray  # [J,3]
    joint_traversal_sequence: np.ndarray
    joint_idx_to_config_idx: np.ndarray
    num_configuration_variables: int
    num_joints: int
    num_links: int

    @property
    def joints(self) -> List[MinimalJoint]:
        return [MinimalJoint(int(self.joint_type[j]), self.joint_X_PL_J[j].copy(), j, int(self.joint_parent_link[j]),
                             int(self.joint_child_link[j]), self.joint_axis[j].copy()) for j in range(self.num_joints)]

    @property
    def links(self) -> List[MinimalLink]:
        out = []
        for l in range(self.num_links):
            parent = np.nonzero(self.joint_child_link == l)[0]
            children = np.nonzero(self.joint_parent_link == l)[0].astype(np.int32)
            out.append(MinimalLink(l, int(parent[0]) if len(parent) else -1, children, int(len(children))))
        return out

    @staticmethod
    def from_tree(t: KinematicTree) -> "MinimalKinematicTree":
        if not t._finalized:
            raise RuntimeError("KinematicTree is not finalized")
        J = len(t.joints)
        return MinimalKinematicTree(
            joint_type=np.array([j.type for j in t.joints], np.int32).reshape(J),
            joint_X_PL_J=np.array([j.X_PL_J for j in t.joints], np.float32).reshape(J, 4, 4),
            joint_parent_link=np.array([j.parent_link for j in t.joints], np.int32).reshape(J),
            joint_child_link=np.array([j.child_link for j in t.joints], np.int32).reshape(J),
            joint_axis=np.array([j.axis for j in t.joints], np.float32).reshape(J, 3),
            joint_traversal_sequence=np.array(t.joint_traversal_sequence, np.int32).reshape(J),
            joint_idx_to_config_idx=np.array(t.joint_idx_to_config_idx, np.int32).reshape(J),
            num_configuration_variables=t.num_configuration_variables,
            num_joints=J,
            num_links=len(t.links),
        )


@dataclass
class SceneInspector:
    link_index_to_scene_collision_geometry_indices: List[List[int]] = field(default_factory=list)
    scene_collision_geometry_name_to_geometry_index: Dict[str, int] = field(default_factory=dict)
    robot_to_world_collision_pairs: List[Tuple[int, int]] = field(default_factory=list)
    robot_geometry_ids: List[int] = field(default_factory=list)

    def get_collision_pair_matrix(self) -> np.ndarray:
        """2 x P int32 (collision_geometry.h:71-82)."""
        m = np.zeros((2, len(self.robot_to_world_collision_pairs)), np.int32)
        for c, (a, b) in enumerate(self.robot_to_world_collision_pairs):
            m[0, c], m[1, c] = a, b
        return m

    getCollisionPairMatrix = get_collision_pair_matrix


class MinimalPlant:
    """Kinematic tree + scene geometries + collision pairs (minimal_plant.h:16-39)."""

    def __init__(self, kin_tree: MinimalKinematicTree, geometries: List[CollisionGeometry],
                 collision_pairs: np.ndarray):
        self.kin_tree = kin_tree
        self.scene_collision_geometries = list(geometries)
        cp = np.asarray(collision_pairs, np.int32).reshape(2, -1)
        self._pairs = np.ascontiguousarray(cp)
        self._arrays = None

    @staticmethod
    def from_arrays(a: Dict[str, np.ndarray], num_configuration_variables: int, num_links: int) -> "MinimalPlant":
        """Rebuild a plant from the flat tables of ``arrays()``."""
        J = int(np.asarray(a["joint_type"]).size)
        kt = MinimalKinematicTree(
            joint_type=np.asarray(a["joint_type"], np.int32).reshape(J),
            joint_X_PL_J=np.asarray(a["joint_X_PL_J"], np.float32).reshape(J, 4, 4).transpose(0, 2, 1).copy(),
            joint_parent_link=np.asarray(a["joint_parent_link"], np.int32).reshape(J),
            joint_child_link=np.asarray(a["joint_child_link"], np.int32).reshape(J),
            joint_axis=np.asarray(a["joint_axis"], np.float32).reshape(J, 3),
            joint_traversal_sequence=np.asarray(a["joint_traversal_sequence"], np.int32).reshape(J),
            joint_idx_to_config_idx=np.asarray(a["joint_idx_to_config_idx"], np.int32).reshape(J),
            num_configuration_variables=int(num_configuration_variables), num_joints=J, num_links=int(num_links))
        G = int(np.asarray(a["geom_type"]).size)
        dims = np.asarray(a["geom_dimensions"], np.float32).reshape(G, 3)
        xlb = np.asarray(a["geom_X_L_B"], np.float32).reshape(G, 4, 4).transpose(0, 2, 1)
        geoms = [CollisionGeometry(type=int(a["geom_type"][g]), dimensions=dims[g].copy(),
                                   link_index=int(a["geom_link_index"][g]), group=int(a["geom_group"][g]),
                                   X_L_B=xlb[g].copy()) for g in range(G)]
        pairs = np.asarray(a["collision_pairs_flat"], np.int32).reshape(-1, 2).T
        return MinimalPlant(kt, geoms, pairs)

    @property
    def num_scene_geometries(self) -> int:
        return len(self.scene_collision_geometries)

    @property
    def num_collision_pairs(self) -> int:
        return int(self._pairs.shape[1])

    @property
    def collision_pairs_flat(self) -> np.ndarray:
        return np.ascontiguousarray(self._pairs.T).reshape(-1)

    def collision_pair_matrix(self) -> np.ndarray:
        return self._pairs.copy()

    def set_collision_pairs_from_matrix(self, m: np.ndarray) -> None:
        m = np.asarray(m, np.int32)
        if m.ndim != 2 or m.shape[0] != 2:
            raise RuntimeError("Matrix must be shape (2, N)")
        self._pairs = np.ascontiguousarray(m)
        self._arrays = None

    def arrays(self) -> Dict[str, np.ndarray]:
        """Contiguous tables in the flat C-ABI layout (4x4 matrices column-major)."""
        if self._arrays is None:
            kt = self.kin_tree
            G = self.num_scene_geometries
            geoms = self.scene_collision_geometries
            self._arrays = dict(
                joint_type=np.ascontiguousarray(kt.joint_type, np.int32),
                joint_parent_link=np.ascontiguousarray(kt.joint_parent_link, np.int32),
                joint_child_link=np.ascontiguousarray(kt.joint_child_link, np.int32),
                joint_idx_to_config_idx=np.ascontiguousarray(kt.joint_idx_to_config_idx, np.int32),
                joint_traversal_sequence=np.ascontiguousarray(kt.joint_traversal_sequence, np.int32),
                joint_X_PL_J=np.ascontiguousarray(
                    np.transpose(kt.joint_X_PL_J, (0, 2, 1)).reshape(-1), np.float32),
                joint_axis=np.ascontiguousarray(kt.joint_axis.reshape(-1), np.float32),
                geom_type=np.array([g.type for g in geoms], np.int32).reshape(G),
                geom_link_index=np.array([g.link_index for g in geoms], np.int32).reshape(G),
                geom_group=np.array([g.group for g in geoms], np.int32).reshape(G),
                geom_dimensions=np.array([np.asarray(g.dimensions, np.float32) for g in geoms],
                                         np.float32).reshape(-1),
                geom_X_L_B=np.array([np.asarray(g.X_L_B, np.float32).T.reshape(-1) for g in geoms],
                                    np.float32).reshape(-1),
                collision_pairs_flat=np.ascontiguousarray(self.collision_pairs_flat, np.int32),
            )
        return self._arrays


class Plant:
    """Plant (minimal_plant.h:42-145): a kinematic tree, its scene inspector and
    the scene's collision geometries, with the reference's accessors.
    numJoints() returns the number of joints (the reference returns the number
    of links there, minimal_plant.h:50)."""

    def __init__(self, kin_tree: KinematicTree, inspector: SceneInspector,
                 scene_collision_geometries: List[CollisionGeometry]):
        self._tree = kin_tree
        self._inspector = inspector
        self._geoms = list(scene_collision_geometries)

    def numLinks(self) -> int:
        return self._tree.numLinks()

    def numJoints(self) -> int:
        return self._tree.numJoints()

    def getPositionLowerLimits(self) -> np.ndarray:
        return self._tree.getPositionLowerLimits()

    def getPositionUpperLimits(self) -> np.ndarray:
        return self._tree.getPositionUpperLimits()

    def numConfigurationVariables(self) -> int:
        return self._tree.numConfigurationVariables()

    def getMinimalPlant(self) -> "MinimalPlant":
        if not self._tree._finalized:
            self._tree.finalize()
        return MinimalPlant(self._tree.get_minimal_kinematic_tree(), self._geoms,
                            self._inspector.get_collision_pair_matrix())

    def getKinematicTree(self) -> KinematicTree:
        return self._tree

    def getSceneInspector(self) -> SceneInspector:
        return self._inspector

    def getRobotGeometryIds(self) -> List[int]:
        return self._inspector.robot_geometry_ids

    def getSceneCollisionGeometries(self) -> List[CollisionGeometry]:
        return self._geoms

    def getCollisionPairMatrix(self) -> np.ndarray:
        return self._inspector.get_collision_pair_matrix()

    def getSceneCollisionGeometryNames(self) -> List[str]:
        names = self._inspector.scene_collision_geometry_name_to_geometry_index
        keys = [""] * len(names)
        for name, idx in names.items():
            keys[idx] = name
        return keys

    def getSceneCollisionGeometryIndexByName(self, name: str) -> int:
        idx = self._inspector.scene_collision_geometry_name_to_geometry_index.get(name)
        if idx is None:
            raise IndexError("Geometry name not found: " + name)
        return idx


# --------------------------------------------------------------------------- scene rules
def _group_geometries(tree: KinematicTree, geoms: List[CollisionGeometry]) -> None:
    """ROBOT unless the geometry reaches the world link through fixed joints only
    (urdf_parser.cpp:507-531)."""
    for g in geoms:
        pj = tree.links[g.link_index].parent_joint
        if pj < 0:
            raise RuntimeError("collision geometry attached to the world link is not supported")
        joint = tree.joints[pj]
        while True:
            if joint.type != JointType.FIXED:
                g.group = CollisionGroup.ROBOT
                break
            if joint.parent_link == 0:
                g.group = CollisionGroup.WORLD
                break
            prev = tree.links[joint.parent_link].parent_joint
            if prev == -1:
                raise RuntimeError("The kinematic tree appears to be disconnected.")
            joint = tree.joints[prev]


def _path_all_fixed(tree: KinematicTree, a: int, b: int, depth: List[int]) -> bool:
    """True if the unique tree path between links a and b uses fixed joints only
    (urdf_parser.cpp:584-601 restated with parent pointers instead of BFS)."""
    all_fixed = True
    while a != b:
        if depth[a] >= depth[b]:
            j = tree.links[a].parent_joint
            a = tree.joints[j].parent_link
        else:
            j = tree.links[b].parent_joint
            b = tree.joints[j].parent_link
        if tree.joints[j].type != JointType.FIXED:
            all_fixed = False
    return all_fixed


def compute_collision_pairs(tree: KinematicTree, geoms: List[CollisionGeometry]) -> List[Tuple[int, int]]:
    """Pair filter of urdf_parser.cpp:546-613: every (A<B) pair with at least one
    robot geometry, excluding same-link, parent/child ("successive") links and
    links connected by fixed joints only. Vectorised over geometry pairs; the
    fixed-path test is tabulated per link pair."""
    n = len(tree.links)
    depth = [0] * n
    for j in tree.joint_traversal_sequence:
        jt = tree.joints[j]
        depth[jt.child_link] = depth[jt.parent_link] + 1
    G = len(geoms)
    if G < 2:
        return []
    link = np.array([g.link_index for g in geoms], np.int64)
    world = np.array([g.group == CollisionGroup.WORLD for g in geoms])
    parent_of = np.array([tree.joints[tree.links[g.link_index].parent_joint].parent_link
                          if tree.links[g.link_index].parent_joint >= 0 else -1 for g in geoms], np.int64)
    used = sorted(set(link.tolist()))
    fixed = np.zeros((n, n), bool)
    for la in used:
        for lb in used:
            fixed[la, lb] = _path_all_fixed(tree, la, lb, depth)
    ia, ib = np.triu_indices(G, k=1)
    la, lb = link[ia], link[ib]
    keep = ~(world[ia] & world[ib])
    keep &= (parent_of[ia] != lb) & (parent_of[ib] != la)
    keep &= la != lb
    keep &= ~fixed[la, lb]
    return list(zip(ia[keep].tolist(), ib[keep].tolist()))


def build_plant(tree: KinematicTree, geoms: List[CollisionGeometry],
                names: Optional[Dict[str, int]] = None) -> Tuple[MinimalPlant, SceneInspector]:
    """finalize_scene + getMinimalPlant for a finalized tree (urdf_parser.cpp:167-206, 485-616)."""
    if not tree._finalized:
        tree.finalize()
    _group_geometries(tree, geoms)
    insp = SceneInspector()
    insp.link_index_to_scene_collision_geometry_indices = [[] for _ in tree.links]
    for i, g in enumerate(geoms):
        insp.link_index_to_scene_collision_geometry_indices[g.link_index].append(i)
    insp.robot_geometry_ids = [i for i, g in enumerate(geoms) if g.group == CollisionGroup.ROBOT]
    insp.robot_to_world_collision_pairs = compute_collision_pairs(tree, geoms)
    insp.scene_collision_geometry_name_to_geometry_index = dict(names or {})
    plant = MinimalPlant(tree.get_minimal_kinematic_tree(), geoms, insp.get_collision_pair_matrix())
    return plant, insp


# --------------------------------------------------------------------------- URDF
def _floats(s: str, n: int) -> List[float]:
    vals = [float(np.float32(v)) for v in s.split()]
    if len(vals) < n:
        raise RuntimeError(f"expected {n} numbers in '{s}'")
    return vals[:n]


def parse_origin(el: Optional[ET.Element]) -> np.ndarray:
    """urdf_parser.cpp:321-381."""
    if el is None:
        return np.eye(4, dtype=np.float32)
    xyz = el.get("xyz")
    if xyz is None:
        raise RuntimeError("[CSDECOMP:URDFPARSER] no position specified for joint origin")
    t = _floats(xyz, 3)
    rpy = _floats(el.get("rpy"), 3) if el.get("rpy") is not None else [0.0, 0.0, 0.0]
    return make_transform(rpy_to_matrix(*rpy), t)


def parse_collision_geometry(col: ET.Element) -> CollisionGeometry:
    """urdf_parser.cpp:403-466 (capsules accepted)."""
    g = CollisionGeometry()
    o = col.find("origin")
    if o is not None:
        g.X_L_B = parse_origin(o)
    geo = col.find("geometry")
    if geo is not None:
        shape = next(iter(geo), None)
        if shape is None:
            raise RuntimeError("No valid geometry type specified.")
        if shape.tag == "box":
            g.type = ShapePrimitive.BOX
            g.dimensions = np.array(_floats(shape.get("size"), 3), np.float32)
        elif shape.tag == "sphere":
            g.type = ShapePrimitive.SPHERE
            g.dimensions = np.array([float(shape.get("radius")), -1, -1], np.float32)
        elif shape.tag == "cylinder":
            raise RuntimeError("cylider not yet implemented")
        elif shape.tag == "capsule":
            r, ln = float(shape.get("radius")), float(shape.get("length"))
            g.type = ShapePrimitive.CAPSULE
            g.dimensions = np.array([r, ln, r], np.float32)
    return g


class URDFParser:
    """URDF / Drake-directive loader with the reference parser's semantics."""

    def __init__(self):
        self.kinematic_tree = KinematicTree()
        self.scene_collision_geometries: List[CollisionGeometry] = []
        self.names: Dict[str, int] = {}
        self.inspector = SceneInspector()
        self.packages: Dict[str, str] = {}
        self._plant: Optional[MinimalPlant] = None

    def register_package(self, name: str, path: str) -> bool:
        if not name or not path or not os.path.exists(path):
            return False
        self.packages[name] = path
        return True

    registerPackage = register_package

    def _resolve(self, path: str) -> str:
        if path.startswith("package://"):
            rest = path[len("package://"):]
            pkg, _, rel = rest.partition("/")
            if pkg in self.packages:
                return os.path.join(self.packages[pkg], rel)
        return path

    def parse_urdf(self, path: str) -> bool:
        with open(path) as f:
            return self.parse_urdf_string(f.read())

    parseURDF = parse_urdf

    def parse_urdf_string(self, text: str) -> bool:
        root = ET.fromstring(text)
        if root.tag != "robot":
            return False
        tree = self.kinematic_tree
        tree.add_link(Link(name="world"))
        for link_el in root.findall("link"):
            self._parse_link(link_el)
        for joint_el in root.findall("joint"):
            self._parse_joint(joint_el)
        if not any(j.parent_link == 0 for j in tree.joints):
            raise RuntimeError("[CSDECOMP:URDFPARSER] The provided urdf is not connected to the 'world' link")
        for link in tree.links[1:]:  # urdf_parser.cpp:136-154
            if link.parent_joint < 0:
                raise RuntimeError(f"[CSDECOMP:URDFPARSER] The link {link.name} has no parent joint; every model "
                                   "must be connected to the world frame.")
        tree.finalize()
        self.finalize_scene()
        return True

    parseURDFString = parse_urdf_string

    def _parse_link(self, el: ET.Element) -> None:
        name = el.get("name")
        if el.get("origin") is not None:
            raise RuntimeError("Global origin tags are not supported in links")
        idx = self.kinematic_tree.add_link(Link(name=name))
        n = 0
        for col in el.findall("collision"):
            if col.get("name") is not None:
                cname = col.get("name") + f"::{n + 1}"
            else:
                cname = name + f"::col_geom::{n + 1}"
            g = parse_collision_geometry(col)
            g.link_index = idx
            self.names[cname] = len(self.scene_collision_geometries)
            self.scene_collision_geometries.append(g)
            n += 1

    def _parse_joint(self, el: ET.Element) -> None:
        tstr = el.get("type")
        types = {"fixed": JointType.FIXED, "revolute": JointType.REVOLUTE, "prismatic": JointType.PRISMATIC}
        if tstr not in types:
            raise RuntimeError(f"Unsupported joint type: {tstr}")
        jt = types[tstr]
        axis = np.zeros(3, np.float32)
        if jt != JointType.FIXED:
            ax = el.find("axis")
            if ax is None:
                raise RuntimeError("revolute or prismatic joint without axis")
            axis = unit_axis(_floats(ax.get("xyz"), 3))
        parent, child = el.find("parent"), el.find("child")
        if parent is None or child is None:
            raise RuntimeError("Joint is missing parent or child element")
        tree = self.kinematic_tree
        j = Joint(name=el.get("name"), type=jt, X_PL_J=parse_origin(el.find("origin")),
                  parent_link=tree.get_link_index(parent.get("link")),
                  child_link=tree.get_link_index(child.get("link")), axis=axis)
        lim = el.find("limit")
        if lim is not None:
            j.position_lower_limit = float(lim.get("lower", 0.0))
            j.position_upper_limit = float(lim.get("upper", 0.0))
        tree.add_joint(j)

    def finalize_scene(self) -> None:
        plant, insp = build_plant(self.kinematic_tree, self.scene_collision_geometries, self.names)
        self._plant, self.inspector = plant, insp

    # directives: urdf_parser.cpp:618-778
    def parse_directives_to_urdf_string(self, path: str) -> str:
        import yaml

        class _Loader(yaml.SafeLoader):
            pass

        _Loader.add_multi_constructor("!", lambda loader, suffix, node: loader.construct_mapping(node))
        with open(path) as f:
            cfg = yaml.load(f, Loader=_Loader)
        out = ['<robot name="combined_robot">']
        for d in cfg["directives"]:
            if "add_model" in d:
                m = d["add_model"]
                root = ET.parse(self._resolve(m["file"])).getroot()
                self._rename(root, m["name"])
                for el in root:
                    out.append(ET.tostring(el, encoding="unicode"))
            elif "add_weld" in d:
                w = d["add_weld"]
                out.append(f'<joint name="weld_{w["parent"]}_to_{w["child"]}" type="fixed">'
                           f'<parent link="{w["parent"]}"/><child link="{w["child"]}"/></joint>')
            elif "add_frame" in d:
                fr = d["add_frame"]
                X = fr["X_PF"]
                t = [float(v) for v in X["translation"]]
                deg = [float(v) for v in X["rotation"]["deg"]]
                rpy = [v * math.pi / 180.0 for v in deg]
                out.append(f'<link name="{fr["name"]}"/>')
                out.append(f'<joint name="{X["base_frame"]}_to_{fr["name"]}" type="fixed">'
                           f'<parent link="{X["base_frame"]}"/><child link="{fr["name"]}"/>'
                           f'<origin xyz="{t[0]:.6g} {t[1]:.6g} {t[2]:.6g}" '
                           f'rpy="{rpy[0]:.6g} {rpy[1]:.6g} {rpy[2]:.6g}"/></joint>')
        out.append("</robot>")
        return "\n".join(out)

    parseDirectivesToURDFString = parse_directives_to_urdf_string

    def _rename(self, el: ET.Element, prefix: str) -> None:
        if el.get("name") is not None:
            el.set("name", f"{prefix}::{el.get('name')}")
        if el.tag == "joint":
            p, c = el.find("parent"), el.find("child")
            if p is not None and p.get("link") is not None:
                if p.get("link") == "world":
                    raise RuntimeError("Directly specifying the world link as parent is not supported")
                p.set("link", f"{prefix}::{p.get('link')}")
            if c is not None and c.get("link") is not None:
                c.set("link", f"{prefix}::{c.get('link')}")
        for ch in el:
            self._rename(ch, prefix)

    def parse_directives(self, path: str) -> bool:
        s = self.parse_directives_to_urdf_string(path)
        if not s:
            return False
        return self.parse_urdf_string(s)

    parseDirectives = parse_directives

    def get_minimal_plant(self) -> MinimalPlant:
        if self._plant is None:
            raise RuntimeError("No URDF has been parsed yet")
        return self._plant

    # urdf_parser.h:116-131, urdf_parser.cpp:477-483
    def override_kinematic_tree(self, kinematic_tree: KinematicTree) -> None:
        self.kinematic_tree = kinematic_tree

    def override_scene_collision_geometries(self, geometries: List[CollisionGeometry]) -> None:
        self.scene_collision_geometries = list(geometries)

    def build_plant(self) -> "Plant":
        if not self.kinematic_tree.is_finalized():
            raise RuntimeError("No URDF has been parsed yet, cannot build plant!")
        return Plant(self.kinematic_tree, self.inspector, self.scene_collision_geometries)

    overrideKinematicTree = override_kinematic_tree
    overrideSceneCollisionGeometries = override_scene_collision_geometries
    buildPlant = build_plant

    getMinimalPlant = get_minimal_plant

    def get_kinematic_tree(self) -> KinematicTree:
        return self.kinematic_tree

    getKinematicTree = get_kinematic_tree

    def get_scene_inspector(self) -> SceneInspector:
        return self.inspector

    getSceneInspector = get_scene_inspector

    def get_scene_collision_geometries(self) -> List[CollisionGeometry]:
        return self.scene_collision_geometries

    def get_minimal_kinematic_tree(self) -> MinimalKinematicTree:
        return self.kinematic_tree.get_minimal_kinematic_tree()
