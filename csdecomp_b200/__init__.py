"""csdecomp_b200 -- B200 (sm_100a) implementation of CSDecomp's hot path.

Batched forward kinematics and primitive-pair collision checks over a
MinimalPlant, batched edge checks, hit-and-run sampling in H-polytopes and
EI-ZO edge inflation and region editing, behind the reference's Python names (see api.py) and
the C ABI of include/csd_capi.h.
"""
from .plant import (CollisionGeometry, CollisionGroup, Joint, JointType, KinematicTree, Link, MinimalJoint,
                    MinimalKinematicTree, MinimalLink, MinimalPlant, Plant, SceneInspector, ShapePrimitive, URDFParser)
from .api import (MAX_DIM, BatchedEdgeInflator, MAX_NUM_FACES, MAX_NUM_VOXELS, CheckCollisionFree, CheckCollisionFreeCuda,
                  CheckCollisionFreeVoxels, CheckCollisionFreeVoxelsCuda, CheckEdgeCollisionFree,
                  CheckEdgesCollisionFreeCuda, CheckEdgesCollisionFreeRankedCuda, ComputeForwardKinematicsCuda, CudaEdgeInflator, EditRegionsCuda,
                  EditRegionsOptions, EizoCuda, EizoInfo,
                  EizoIterationInfo, EizoOptions, HPolyhedron, MinimalHPolyhedron, PairCollisionFree, Voxels,
                  UniformSampleInHPolyhedraCuda, VisibilityGraph, computeLinkFrameToWorldTransformsMinimal,
                  numSamplesUnadaptive,
                  plant_handle, printEizoSummary)
from ._capi import CSD_EDGE_L2_REF, CSD_EDGE_LINF, CSD_EDGE_VG, CsdError, NativeURDFParser

__all__ = [n for n in dir() if not n.startswith("_")]
