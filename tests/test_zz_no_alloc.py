"""Allocation-free EI-ZO entry point (csd_eizo_noalloc).

Some callers cannot allocate device memory while they run: a real-time
planning loop that owns a fixed memory budget, or a host process that forbids
allocation after start-up. csd_eizo_noalloc serves them from a fixed array in
the library's static device memory. This test calls it through the C ABI and
checks it returns the same region as csd_eizo, bit for bit, on two calls in a
row (the second call reuses the array the first one left behind), that free
device memory is unchanged across a call, and the same with voxels. The file
is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import csdecomp_b200 as csd
from csdecomp_b200 import _capi as C
from csdecomp_b200 import scenes
from csdecomp_b200.plant import ShapePrimitive

pytestmark = pytest.mark.gpu


def _call(fn, h, ls, le, A0, b0, ids, opt, cap, noalloc, voxels=None, vr=0.0):
    d = ls.size
    A = np.zeros((cap, d), np.float32)
    b = np.zeros(cap, np.float32)
    info = (C.EizoIterC * int(opt.max_iterations))()
    nf, nit = ctypes.c_int32(0), ctypes.c_int32(0)
    o = opt._c()
    nv = 0 if voxels is None else voxels.shape[0]
    args = [h.handle, C.ptr(ls), C.ptr(le), C.ptr(voxels) if nv else None, nv, ctypes.c_float(vr), C.ptr(A0),
            C.ptr(b0), A0.shape[0], C.ptr(ids), ids.size, ctypes.byref(o), cap, C.ptr(A), C.ptr(b), ctypes.byref(nf),
            info, len(info), ctypes.byref(nit)]
    if noalloc:
        args.append(None)
    C.check(fn(*args))
    return A[:nf.value].copy(), b[:nf.value].copy(), [info[i].num_faces_placed for i in range(nit.value)]


def _edges_and_domain(sc):
    q = sc.random_configs(4000, 23)
    free = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1]
    edges = []
    for q0 in free:
        q1 = np.clip(q0 + 0.2, -3.1, 3.1).astype(np.float32)
        if csd.CheckEdgeCollisionFree(q0, q1, sc.plant):
            edges.append((np.ascontiguousarray(q0), q1))
        if len(edges) == 2:
            break
    assert len(edges) == 2
    dom = csd.HPolyhedron()
    dom.MakeBox(sc.lower(), sc.upper())
    return edges, np.ascontiguousarray(dom.A(), np.float32), np.ascontiguousarray(dom.b(), np.float32)


def test_noalloc_matches_eizo_twice():
    sc = scenes.edge_check_scene(keepout=0.8)
    edges, A0, b0 = _edges_and_domain(sc)
    ids = np.ascontiguousarray(sc.inspector.robot_geometry_ids, np.int32)
    opt = csd.EizoOptions(num_particles=1000, mixing_steps=30, max_iterations=50)
    h = csd.plant_handle(sc.plant)
    for ls, le in edges:  # two calls in a row
        ref = _call(C.lib().csd_eizo, h, ls, le, A0, b0, ids, opt, 1000, False)
        free_before = torch.cuda.mem_get_info()[0]
        got = _call(C.lib().csd_eizo_noalloc, h, ls, le, A0, b0, ids, opt, 1000, True)
        assert torch.cuda.mem_get_info()[0] == free_before  # no device memory taken by the call
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
        assert got[2] == ref[2]
        assert ref[0].shape[0] > A0.shape[0]


def test_noalloc_with_voxels_matches_eizo_twice():
    """Voxels checked against robot geometry ids that name moving spheres and
    capsules (the two voxel tables of the fused check): csd_eizo, which
    buckets the voxels in a hash grid, and csd_eizo_noalloc, which tests every
    voxel, place the same faces bit for bit, on two calls in a row."""
    sc = scenes.edge_check_scene(keepout=0.8)
    edges, A0, b0 = _edges_and_domain(sc)
    rng = np.random.default_rng(7)
    v = rng.normal(size=(600, 3))
    v = (v / np.linalg.norm(v, axis=1, keepdims=True) * rng.uniform(0.55, 1.0, (600, 1))).astype(np.float32)
    vox = np.ascontiguousarray(v)
    types = [int(g.type) for g in sc.plant.scene_collision_geometries]
    rids = list(sc.inspector.robot_geometry_ids)
    caps = [g for g in rids if types[g] == int(ShapePrimitive.CAPSULE)]
    sph = [g for g in rids if types[g] == int(ShapePrimitive.SPHERE)]
    assert caps and sph
    ids = np.ascontiguousarray(sph[::2] + caps, np.int32)
    opt = csd.EizoOptions(num_particles=800, mixing_steps=20, max_iterations=30)
    h = csd.plant_handle(sc.plant)
    placed = 0
    for ls, le in edges:
        ref = _call(C.lib().csd_eizo, h, ls, le, A0, b0, ids, opt, 1000, False, vox, 0.03)
        got = _call(C.lib().csd_eizo_noalloc, h, ls, le, A0, b0, ids, opt, 1000, True, vox, 0.03)
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
        assert got[2] == ref[2]
        placed += ref[0].shape[0] - A0.shape[0]
    # the voxels change the regions: the same calls without voxels differ
    nov = _call(C.lib().csd_eizo, h, edges[1][0], edges[1][1], A0, b0, ids, opt, 1000, False)
    assert placed > 0 and not (nov[0].shape == ref[0].shape and np.array_equal(nov[0], ref[0]))


def test_noalloc_rejects_oversized_options():
    sc = scenes.point_check_scene()
    dom = csd.HPolyhedron()
    dom.MakeBox(sc.lower(), sc.upper())
    A0 = np.ascontiguousarray(dom.A(), np.float32)
    b0 = np.ascontiguousarray(dom.b(), np.float32)
    ids = np.zeros(0, np.int32)
    ls = np.zeros(7, np.float32)
    opt = csd.EizoOptions(num_particles=1000, epsilon=0.001)  # ~1.3e5 unadaptive samples: too large
    with pytest.raises(csd.CsdError) as ei:
        _call(C.lib().csd_eizo_noalloc, csd.plant_handle(sc.plant), ls, ls, A0, b0, ids, opt, 1000, True)
    assert ei.value.code == C.CSD_ERR_CAPACITY
