"""Allocation-free EI-ZO entry point (csd_eizo_noalloc).

Some callers cannot allocate device memory while they run: a real-time
planning loop that owns a fixed memory budget, or a host process that forbids
allocation after start-up. csd_eizo_noalloc serves them from a fixed array in
the library's static device memory. This test calls it through the C ABI and
checks it returns the same region as csd_eizo, bit for bit, on two calls in a
row (the second call reuses the array the first one left behind). The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import csdecomp_b200 as csd
from csdecomp_b200 import _capi as C
from csdecomp_b200 import scenes

pytestmark = pytest.mark.gpu


def _call(fn, h, ls, le, A0, b0, ids, opt, cap, noalloc):
    d = ls.size
    A = np.zeros((cap, d), np.float32)
    b = np.zeros(cap, np.float32)
    info = (C.EizoIterC * int(opt.max_iterations))()
    nf, nit = ctypes.c_int32(0), ctypes.c_int32(0)
    o = opt._c()
    args = [h.handle, C.ptr(ls), C.ptr(le), None, 0, ctypes.c_float(0.0), C.ptr(A0), C.ptr(b0), A0.shape[0],
            C.ptr(ids), ids.size, ctypes.byref(o), cap, C.ptr(A), C.ptr(b), ctypes.byref(nf), info, len(info),
            ctypes.byref(nit)]
    if noalloc:
        args.append(None)
    C.check(fn(*args))
    return A[:nf.value].copy(), b[:nf.value].copy(), [info[i].num_faces_placed for i in range(nit.value)]


def test_noalloc_matches_eizo_twice():
    sc = scenes.edge_check_scene(keepout=0.8)
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
    A0 = np.ascontiguousarray(dom.A(), np.float32)
    b0 = np.ascontiguousarray(dom.b(), np.float32)
    ids = np.ascontiguousarray(sc.inspector.robot_geometry_ids, np.int32)
    opt = csd.EizoOptions(num_particles=1000, mixing_steps=30, max_iterations=50)
    h = csd.plant_handle(sc.plant)
    for ls, le in edges:  # two calls in a row
        ref = _call(C.lib().csd_eizo, h, ls, le, A0, b0, ids, opt, 1000, False)
        got = _call(C.lib().csd_eizo_noalloc, h, ls, le, A0, b0, ids, opt, 1000, True)
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
        assert got[2] == ref[2]
        assert ref[0].shape[0] > A0.shape[0]


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
