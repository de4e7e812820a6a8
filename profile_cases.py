"""Small, reproducible launches of the hot kernels for profiler captures.

  python profile_cases.py check_points [--configs N] [--no-cull]
      one warm-up and one timed check_points launch on N collision-free
      configurations of the 7-DOF arm (80 spheres + 4 capsules) in 200 world
      primitives (with --no-cull every pair is evaluated: the full sweep)
  python profile_cases.py batch [--slots S] [--iterations I] [--dim {7,14}]
      [--sample-variant V] [--check-item-cap C] [--per-iteration] [--surrogate]
      S inflations of the batched EI-ZO workload (first S scenes), at most I
      iterations, launched stage by stage (profiling mode) with the given
      sampler variant and check work-item cap (defaults: the shapes the
      autotuner picks on a B200; --sample-variant -1: a first call autotunes
      over its first 4 iterations, with the variant switch on region growth,
      and a second call on the same inputs is profiled)

  python profile_cases.py point_check [--configs N]
      config 1: 7-DOF arm, 40 spheres, 20 world boxes; N uniform configurations
  python profile_cases.py edge_check [--edges E]
      config 2: 7-DOF arm, 80 spheres + 4 capsules, 200 world primitives; E
      segments with endpoints uniform in the joint limits, 0.01 rad step
  python profile_cases.py eizo_single [--regions R]
      config 3: R single inflations (CudaEdgeInflator) on the 7-DOF /
      200-primitive scene, seed edges U[0.1, 0.5] rad

  python profile_cases.py visibility_graph [--nodes n]
      VisibilityGraph over n free configurations of the config-3 scene, 0.01 rad
      step (n (n - 1) / 2 edges checked on the device)
  python profile_cases.py voxel_check [--configs N] [--voxels V]
      checkCollisionFreeVoxelsCuda at scale: the config-2 arm (80 spheres + 4
      capsules, 200 world primitives) against V voxels of radius 0.02 m
      (uniform in a 3 x 3 x 1.5 m box around the arm, none within 0.9 m of its
      base, so that verdicts are mixed), N uniform configurations; with and
      without the voxel hash grid
  python profile_cases.py edge_check_ranked [--edges E]
      config-2 arm with a 0.8 m keep-out (mixed verdicts): E edges from free
      starts, lengths U[0.05, 1.0] rad; unranked checks against checks ranked
      by a surrogate trained on 65,536 labelled configurations of the scene
  python profile_cases.py edit_regions [--regions R] [--collisions C]
      EditRegionsCuda on the config-3 scene: R box regions around seed edges,
      C colliding configurations drawn inside each, 9 bisection steps

  python profile_cases.py mlp [--nets K] [--rows R] [--train-steps T]
      surrogate bank of K 14-input nets: T Adam steps of 512 rows per net
      (tensor-core backward GEMMs) and one scoring pass of R rows per net
      (fused tensor-core forward)

Each prints the device time of what it ran (CUDA events, after one warm-up).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def check_points(n: int, cull: bool = True) -> None:
    import torch
    import csdecomp_b200 as csd
    from csdecomp_b200 import _capi as C
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene(keepout=0.8)
    h = csd.plant_handle(sc.plant)
    q = sc.random_configs(200000, 77)
    free = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1]
    h.set_culling(cull)
    qf = np.ascontiguousarray(np.tile(free, (int(np.ceil(n / len(free))), 1))[:n])
    tq = torch.from_numpy(qf).cuda()
    out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()
    ms = []
    for _ in range(2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        C.check(C.lib().csd_check_points(h.handle, C.ptr(tq.data_ptr()), ctypes.c_int64(n), None, 0,
                                         ctypes.c_float(0), None, 0, C.ptr(out.data_ptr()), C.CSD_PTR_DEVICE,
                                         ctypes.c_void_p(st.cuda_stream)))
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    assert int(out.sum().item()) == n
    print(json.dumps({"case": "check_points", "configs": n, "broad_phase": cull,
                      "flop_per_config": h.flops()["total"], "launch_ms": ms[-1]}))


def batch(slots: int, iterations: int, sample_variant: int, check_item_cap: int, per_iteration: bool = False,
          dim: int = 0, surrogate: bool = False) -> None:
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    eizo = dict(num_particles=2000, mixing_steps=50, bisection_steps=9, max_hyperplanes_per_iteration=10,
                epsilon=0.01, delta=0.05, tau=0.5, max_iterations=iterations, configuration_margin=0.01, seed=1337)
    scs, edges = [], []
    seeds = scenes.batch_scene_seeds(4 * slots + 64)
    for i, s in enumerate(seeds):
        if dim and (7 if i % 2 == 0 else 14) != dim:
            continue
        sc = scenes.batch_scene(i, s)
        e = scenes.seed_edges(sc, 1, 3000 + 101 * i, lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                              lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant))
        if e:
            scs.append(sc)
            edges.append(e[0])
        if len(scs) == slots:
            break
    doms = []
    for sc in scs:
        d = csd.HPolyhedron()
        d.MakeBox(sc.lower(), sc.upper())
        doms.append(d)
    b = csd.BatchedEdgeInflator([sc.plant for sc in scs], csd.EizoOptions(**eizo), max_slots=len(scs),
                                face_capacity=4000, autotune_iterations=0 if sample_variant >= 0 else 4)
    if sample_variant >= 0:
        b.set_shapes(sample_variant, check_item_cap)
    if surrogate:  # one net per scene, 16,384 exact labels each, 2 epochs (the benchmark trains 6)
        from csdecomp_b200.surrogate import CollisionSurrogate, training_set
        data = [training_set(sc, [e], 16384, seed=5000 + i) for i, (sc, e) in enumerate(zip(scs, edges))]
        bank = CollisionSurrogate([sc.dim for sc in scs], seed=5000)
        bank.train([x for x, _ in data], [y for _, y in data], batch=512, epochs=2, lr=2e-3)
        b.set_surrogate(bank, 0.01)
    if sample_variant < 0:  # a first call tunes (as the benchmark's warm-up step does); the second is profiled
        b.inflate(list(range(len(scs))), [e[0] for e in edges], [e[1] for e in edges], doms)
    b.set_profiling(True)
    b.inflate(list(range(len(scs))), [e[0] for e in edges], [e[1] for e in edges], doms)
    out = {"case": "batch", "slots": len(scs), "stage_ms": b.stage_ms(), "iterations": b.last_iterations.tolist(),
           "sample_flop": b.sample_flops(),
           "sample_variant": b.SAMPLE_VARIANTS[sample_variant] if sample_variant >= 0 else b.tuning()}
    if per_iteration:
        ms, act = b.iteration_profile()
        var, faces = b.iteration_variants()
        out["per_iteration"] = {"active": act.tolist(), "total_ms": ms.sum(1).round(3).tolist(),
                                "stages": list(b.STAGES), "stage_ms": ms.round(3).tolist(),
                                "variant": var.tolist(), "max_faces": faces.tolist()}
    print(json.dumps(out))


def mlp(nets: int, rows: int, steps: int) -> None:
    """Surrogate bank of `nets` 14-input nets: `steps` Adam steps of 512 rows
    per net (backward GEMMs, gemm_kernel) and one scoring pass of `rows` rows
    per net (fused forward, mlp_forward_kernel), each timed after a warm-up."""
    import torch
    from csdecomp_b200.surrogate import CollisionSurrogate
    rng = np.random.default_rng(3)
    bank = CollisionSurrogate([14] * nets, seed=1)
    xs = [rng.uniform(-np.pi, np.pi, (rows, 14)).astype(np.float32) for _ in range(nets)]
    ys = [(np.linalg.norm(x, axis=1) < 5.0).astype(np.uint8) for x in xs]
    t_train, _ = _timed(lambda: bank.train(xs, ys, batch=512, epochs=512 * steps / rows, lr=1e-3), reps=2)
    t_fwd, _ = _timed(lambda: bank.logits(list(enumerate(xs))), reps=3)
    fwd_flop = 2.0 * nets * rows * (16 * 256 + 2 * 256 * 256 + 256)
    print(json.dumps({"case": "mlp", "nets": nets, "rows_per_net": rows, "train_steps": steps,
                      "train_ms": t_train, "forward_ms": t_fwd, "forward_flop": fwd_flop,
                      "forward_tflops_incl_copies": fwd_flop / t_fwd / 1e9}))


def _timed(fn, reps: int = 3):
    import torch
    fn()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        out = fn()
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best, out


def point_check(n: int) -> None:
    import torch
    import csdecomp_b200 as csd
    from csdecomp_b200 import _capi as C
    from csdecomp_b200 import scenes
    sc = scenes.point_check_scene()
    h = csd.plant_handle(sc.plant)
    q = torch.from_numpy(np.ascontiguousarray(sc.random_configs(n, 5))).cuda()
    out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()

    def run():
        C.check(C.lib().csd_check_points(h.handle, C.ptr(q.data_ptr()), ctypes.c_int64(n), None, 0,
                                         ctypes.c_float(0), None, 0, C.ptr(out.data_ptr()), C.CSD_PTR_DEVICE,
                                         ctypes.c_void_p(st.cuda_stream)))
    ms, _ = _timed(run)
    print(json.dumps({"case": "point_check", "configs": n, "ms": ms, "configs_per_s": n / ms * 1e3,
                      "free_fraction": float(out.float().mean().item())}))


def edge_check(n: int) -> None:
    import torch
    import csdecomp_b200 as csd
    from csdecomp_b200 import _capi as C
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene()
    h = csd.plant_handle(sc.plant)
    a = torch.from_numpy(np.ascontiguousarray(sc.random_configs(n, 6))).cuda()
    b = torch.from_numpy(np.ascontiguousarray(sc.random_configs(n, 7))).cuda()
    out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    pts = torch.zeros(n, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream()

    def run():
        C.check(C.lib().csd_check_edges(h.handle, C.ptr(a.data_ptr()), C.ptr(b.data_ptr()), ctypes.c_int64(n),
                                        ctypes.c_float(0.01), C.CSD_EDGE_L2_REF, C.ptr(out.data_ptr()),
                                        C.ptr(pts.data_ptr()), C.CSD_PTR_DEVICE, ctypes.c_void_p(st.cuda_stream)))
    ms, _ = _timed(run)
    print(json.dumps({"case": "edge_check", "edges": n, "ms": ms, "edges_per_s": n / ms * 1e3,
                      "free_fraction": float(out.float().mean().item()),
                      "points_checked": int(pts.sum().item())}))


def eizo_single(regions: int) -> None:
    import torch
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene(keepout=0.8)
    edges = scenes.seed_edges(sc, regions + 1, 3000, lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                              lambda x, y: csd.CheckEdgesCollisionFreeCuda(x.T, y.T, sc.plant), length=(0.1, 0.5))
    dom = csd.HPolyhedron()
    dom.MakeBox(sc.lower(), sc.upper())
    opt = csd.EizoOptions(num_particles=2000, mixing_steps=50, bisection_steps=9, max_hyperplanes_per_iteration=10,
                          epsilon=0.01, delta=0.05, tau=0.5, max_iterations=500, configuration_margin=0.01,
                          seed=1337)
    inf = csd.CudaEdgeInflator(sc.plant, sc.inspector.robot_geometry_ids, opt, dom)
    inf.inflateEdge(edges[0][0], edges[0][1], None, 0.0, verbose=False)
    st = torch.cuda.current_stream()
    total, faces = 0.0, 0
    for q0, q1 in edges[1:]:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        P = inf.inflateEdge(q0, q1, None, 0.0, verbose=False)
        e1.record(st)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        faces += P.A().shape[0]
    print(json.dumps({"case": "eizo_single", "regions": regions, "ms": total, "regions_per_s": regions / total * 1e3,
                      "mean_faces": faces / regions}))


def visibility_graph(n: int) -> None:
    import torch
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene(keepout=0.8)
    q = sc.random_configs(8 * n, 21)
    nodes = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1][:n]
    ms, A = _timed(lambda: csd.VisibilityGraph(nodes.T, sc.plant, 0.01), reps=1)
    E = len(nodes) * (len(nodes) - 1) // 2
    print(json.dumps({"case": "visibility_graph", "nodes": len(nodes), "edges": E, "ms": ms,
                      "edges_per_s": E / ms * 1e3, "free_edges": int(A.nnz)}))


def edit_regions(regions: int, per_region: int) -> None:
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene(keepout=0.8)
    edges = scenes.seed_edges(sc, regions, 3100, lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                              lambda x, y: csd.CheckEdgesCollisionFreeCuda(x.T, y.T, sc.plant), length=(0.1, 0.5))
    rng = np.random.default_rng(5)
    lo, hi = sc.lower(), sc.upper()
    doms, cols, segs = [], [], []
    for r, (q0, q1) in enumerate(edges):
        blo = np.maximum(lo, np.minimum(q0, q1) - 1.2).astype(np.float32)
        bhi = np.minimum(hi, np.maximum(q0, q1) + 1.2).astype(np.float32)
        P = csd.HPolyhedron()
        P.MakeBox(blo, bhi)
        doms.append(P)
        got = np.zeros((0, sc.dim), np.float32)
        for _ in range(8):  # bounded: a box may hold few collisions
            q = (blo + (bhi - blo) * rng.random((16 * per_region, sc.dim))).astype(np.float32)
            got = np.concatenate([got, q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 0]])
            if got.shape[0] >= per_region:
                break
        got = got[:per_region]
        cols.append(got)
        segs.append(np.full(got.shape[0], r))
    col = np.concatenate(cols).T
    seg = np.concatenate(segs)
    ls = np.stack([e[0] for e in edges], 1).astype(np.float32)
    le = np.stack([e[1] for e in edges], 1).astype(np.float32)
    opts = csd.EditRegionsOptions()
    rids = sc.inspector.robot_geometry_ids
    ms, out = _timed(lambda: csd.EditRegionsCuda(col, seg, ls, le, doms, sc.plant, rids, csd.Voxels(), 0.01, opts))
    added = sum(e.b().size - d.b().size for e, d in zip(out[0], doms))
    n = col.shape[1]
    print(json.dumps({"case": "edit_regions", "regions": len(edges), "collisions": n, "ms": ms,
                      "collisions_per_s": n / ms * 1e3, "checks_per_s": n * opts.bisection_steps / ms * 1e3,
                      "faces_added": int(added)}))


def voxel_scene(voxels: int, seed: int = 17):
    """The voxel-at-scale workload: (scene, voxels [V][3], radius, robot ids)."""
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene(keepout=0.8)
    rng = np.random.default_rng(seed)
    v = np.zeros((0, 3), np.float32)
    while v.shape[0] < voxels:
        c = rng.uniform([-1.5, -1.5, 0.0], [1.5, 1.5, 1.5], (2 * voxels, 3)).astype(np.float32)
        v = np.concatenate([v, c[np.linalg.norm(c, axis=1) > 0.9]])
    return sc, np.ascontiguousarray(v[:voxels]), 0.02, sc.inspector.robot_geometry_ids


def voxel_check(n: int, voxels: int) -> None:
    import torch
    import csdecomp_b200 as csd
    from csdecomp_b200 import _capi as C
    sc, vox, vr, rids = voxel_scene(voxels)
    h = csd.plant_handle(sc.plant)
    q = torch.from_numpy(np.ascontiguousarray(sc.random_configs(n, 5))).cuda()
    vd = torch.from_numpy(vox).cuda()
    ids = np.ascontiguousarray(np.asarray(list(rids), np.int32))  # robot ids are host memory
    out = torch.zeros(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()

    def run():
        C.check(C.lib().csd_check_points(h.handle, C.ptr(q.data_ptr()), ctypes.c_int64(n), C.ptr(vd.data_ptr()),
                                         voxels, ctypes.c_float(vr), C.ptr(ids), len(rids),
                                         C.ptr(out.data_ptr()), C.CSD_PTR_DEVICE, ctypes.c_void_p(st.cuda_stream)))
    res = {}
    for grid in (True, False):
        h.set_voxel_grid(grid)
        ms, _ = _timed(run)
        res["grid" if grid else "every_voxel"] = {"ms": ms, "configs_per_s": n / ms * 1e3,
                                                   "free_fraction": float(out.float().mean().item())}
    h.set_voxel_grid(True)
    print(json.dumps({"case": "voxel_check", "configs": n, "voxels": voxels, "voxel_radius": vr, **res}))


def edge_check_ranked(n: int) -> None:
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    from csdecomp_b200.surrogate import CollisionSurrogate, training_set
    sc = scenes.edge_check_scene(keepout=0.8)
    seeds = scenes.seed_edges(sc, 64, 77, lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                              lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant))
    bank = CollisionSurrogate([sc.dim], seed=1)
    x, y = training_set(sc, seeds, 65536, seed=2)
    bank.train([x], [y], batch=512, epochs=6, lr=2e-3)
    rng = np.random.default_rng(9)
    q = sc.random_configs(8 * n, 10)
    q0 = q[csd.CheckCollisionFreeCuda(q.T, sc.plant) == 1][:n]
    d = rng.normal(size=q0.shape)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q1 = np.clip(q0 + rng.uniform(0.05, 1.0, (len(q0), 1)) * d, sc.lower(), sc.upper()).astype(np.float32)
    ms_u, (fu, pu) = _timed(lambda: csd.CheckEdgesCollisionFreeCuda(q0.T, q1.T, sc.plant, 0.01,
                                                                  return_points_checked=True))
    ms_r, (fr, pr) = _timed(lambda: csd.CheckEdgesCollisionFreeRankedCuda(q0.T, q1.T, sc.plant, bank, 0, 0.01, top=8,
                                                                        return_points_checked=True))
    col = fu == 0
    print(json.dumps({"case": "edge_check_ranked", "edges": int(len(q0)), "free_fraction": float(fu.mean()),
                      "identical": bool((fu == fr).all()),
                      "unranked": {"ms": ms_u, "points": int(pu.sum()), "points_per_colliding_edge": float(pu[col].mean())},
                      "ranked": {"ms": ms_r, "points": int(pr.sum()), "points_per_colliding_edge": float(pr[col].mean())},
                      "training_colliding_fraction": float(y.mean())}))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["check_points", "batch", "point_check", "edge_check", "eizo_single",
                                     "visibility_graph", "edit_regions", "voxel_check", "edge_check_ranked", "mlp"])
    ap.add_argument("--configs", type=int, default=1 << 20)
    ap.add_argument("--no-cull", action="store_true", help="check_points: link-level broad phase off (full sweep)")
    ap.add_argument("--slots", type=int, default=24)
    ap.add_argument("--edges", type=int, default=100000)
    ap.add_argument("--regions", type=int, default=20)
    ap.add_argument("--nodes", type=int, default=1000)
    ap.add_argument("--collisions", type=int, default=512, help="edit_regions: collisions per region")
    ap.add_argument("--voxels", type=int, default=10000, help="voxel_check: voxels")
    ap.add_argument("--iterations", type=int, default=12)
    ap.add_argument("--sample-variant", type=int, default=1)  # index into SAMPLE_VARIANTS; -1: autotune
    ap.add_argument("--check-item-cap", type=int, default=128)
    ap.add_argument("--per-iteration", action="store_true", help="batch: stage times and active slots per iteration")
    ap.add_argument("--dim", type=int, default=0, choices=[0, 7, 14], help="batch: only 7-DOF or 14-DOF scenes")
    ap.add_argument("--surrogate", action="store_true", help="batch: surrogate-ordered checks (nets trained first)")
    ap.add_argument("--nets", type=int, default=64, help="mlp: nets in the bank")
    ap.add_argument("--rows", type=int, default=16384, help="mlp: rows per net")
    ap.add_argument("--train-steps", type=int, default=32, help="mlp: Adam steps")
    a = ap.parse_args()
    if a.case == "check_points":
        check_points(a.configs, not a.no_cull)
    elif a.case == "point_check":
        point_check(a.configs)
    elif a.case == "edge_check":
        edge_check(a.edges)
    elif a.case == "eizo_single":
        eizo_single(a.regions)
    elif a.case == "visibility_graph":
        visibility_graph(a.nodes)
    elif a.case == "edit_regions":
        edit_regions(a.regions, a.collisions)
    elif a.case == "voxel_check":
        voxel_check(a.configs, a.voxels)
    elif a.case == "edge_check_ranked":
        edge_check_ranked(a.edges)
    elif a.case == "mlp":
        mlp(a.nets, a.rows, a.train_steps)
    else:
        batch(a.slots, a.iterations, a.sample_variant, a.check_item_cap, a.per_iteration, a.dim, a.surrogate)


if __name__ == "__main__":
    main()
