"""GPU hit-and-run against the oracle: bit-identical samples (same
counter-based stream, same operation order)."""
import numpy as np
import pytest

import csdecomp_b200 as csd
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def random_polytope(d, extra, seed):
    rng = np.random.default_rng(seed)
    A = [-np.eye(d), np.eye(d)]
    b = [np.full(d, np.pi), np.full(d, np.pi)]
    for _ in range(extra):
        a = rng.normal(size=d)
        a /= np.linalg.norm(a)
        A.append(a[None])
        b.append(np.array([rng.uniform(0.3, 2.0)]))
    return np.vstack(A).astype(np.float32), np.concatenate(b).astype(np.float32)


@pytest.mark.parametrize("d,extra", [(2, 3), (7, 40), (14, 120)])
def test_bit_exact_vs_oracle(d, extra):
    polys, starts = [], []
    for k in range(3):
        A, b = random_polytope(d, extra, 100 * d + k)
        polys.append(csd.HPolyhedron(A, b))
        starts.append(np.zeros(d, np.float32))
    out = csd.UniformSampleInHPolyhedraCuda(polys, np.array(starts).T, 700, 30, seed=4242)
    for k, p in enumerate(polys):
        ref, nf = O.hit_and_run(p.A(), p.b(), starts[k], 700, 30, seed=4242, stream=k)
        assert nf == 0
        np.testing.assert_array_equal(out[k].T, ref)
        assert (p.A() @ out[k] <= p.b()[:, None] + 1e-5).all()


def test_not_contained_raises():
    A, b = random_polytope(3, 0, 1)
    with pytest.raises(RuntimeError):
        csd.UniformSampleInHPolyhedraCuda([csd.HPolyhedron(A, b)], np.full((3, 1), 5.0, np.float32), 10, 5)


def test_failed_chain_writes_nan_device_pointers():
    torch = pytest.importorskip("torch")
    import ctypes
    from csdecomp_b200 import _capi as C
    A, b = random_polytope(3, 0, 1)
    dev = torch.device("cuda:0")
    tA = torch.from_numpy(A).to(dev)
    tb = torch.from_numpy(b).to(dev)
    off = torch.tensor([0, A.shape[0]], dtype=torch.int32, device=dev)
    # outside the box: a chain fails unless its first direction points back into the box
    start = torch.full((1, 3), 5.0, device=dev)
    S = 64
    out = torch.zeros((1, S, 3), device=dev)
    nf = ctypes.c_int32(-1)
    C.check(C.lib().csd_uniform_sample_hpolyhedra(C.ptr(tA.data_ptr()), C.ptr(tb.data_ptr()),
                                                  C.ptr(off.data_ptr()), 1, 3, C.ptr(start.data_ptr()), S, 4,
                                                  ctypes.c_uint64(1), C.ptr(out.data_ptr()), ctypes.byref(nf),
                                                  C.CSD_PTR_DEVICE, None))
    torch.cuda.synchronize()
    got = out.cpu().numpy()[0]
    ref, ref_nf = O.hit_and_run(A, b, np.full(3, 5.0, np.float32), S, 4, seed=1)
    assert 0 < nf.value < S and nf.value == ref_nf
    assert (np.isnan(got).all(1) == np.isnan(ref).all(1)).all()
    assert int(np.isnan(got).all(1).sum()) == nf.value
    ok = ~np.isnan(ref).all(1)
    np.testing.assert_array_equal(got[ok], ref[ok])


def test_uniformity_in_box():
    d = 7
    p = csd.HPolyhedron()
    p.MakeBox(-np.pi * np.ones(d), np.pi * np.ones(d))
    s = csd.UniformSampleInHPolyhedraCuda([p], np.zeros((d, 1), np.float32), 20000, 50)[0]
    assert np.abs(s.mean(1)).max() < 0.06
    assert np.abs(s.var(1) - np.pi ** 2 / 3).max() < 0.15
