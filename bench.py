#!/usr/bin/env python
"""Benchmark: EI-ZO regions/s and configs/s on one B200, batched form: 256
inflations per step on 256 seeded scenes (7-DOF and 14-DOF plants mixed), the
plain GPU form (one inflation per call) on the same inputs beside it, the
point- and edge-check workloads (configs 1 and 2) and the single-inflation
workload (config 3), the collision kernel's FP32 roofline, and the CPU
oracle's EI-ZO and checks on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]

One step = one BatchedEdgeInflator.inflate of the rank's seed edges, one per
scene. The workload is one fixed list of N x 256 scenes; N > 1 (torchrun)
splits it into contiguous ranges of equal predicted cost (dimension^2 x
primitives), one per rank (weak scaling, no collective on the data path);
rank 0 prints one JSON line.

The CPU sample (reference arm and the GPU arm's cpu_baseline leg) is the same
fixed set of inflations in both arms: scenes 0-3 of the workload (two 7-DOF,
two 14-DOF), each scene's first seed edge, found with the oracle's checker.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "EI-ZO regions/s and configs/s on 1 B200: surrogate+batched vs plain GPU, ε=0.01"
NUM_SLOTS = 256
FACE_CAPACITY = 4000          # hpolyhedron.h:5 default region capacity
EIZO_KW = dict(num_particles=2000, mixing_steps=50, bisection_steps=9, max_hyperplanes_per_iteration=10,
               epsilon=0.01, delta=0.05, tau=0.5, max_iterations=500, configuration_margin=0.01, seed=1337)
WORKLOAD = ("batched EI-ZO: 256 inflations per step per GPU, one per seeded scene (even: 7-DOF arm, 80 spheres + 4 "
            "capsules; odd: 14-DOF two-arm plant, 2 x (40 spheres + 2 capsules)); U{50..400} world primitives per "
            "scene (half boxes, half spheres, centres U[-1,1]^3, 0.8 m keep-out around each base); seed edges "
            "U[0.05,1.0] rad in free space; domain = joint-limit box; 2000 particles, mixing 50, 9 bisection steps, "
            "<=10 faces/iteration, eps=0.01, delta=0.05, tau=0.5, run to admissibility (max 500 iterations); "
            "region capacity 4000 faces (the regions are not capped at 300 faces: see faces)")
L2_RULE = "GPU arm: L2 flushed between steps (256 MB write)"
SEED_EDGE_SEED = 3000
SURROGATE_ROWS = 16384        # labelled configurations per scene (4.2 M over the 256 scenes)
SURROGATE_EPOCHS = 6
SURROGATE_SEED = 5000
SURROGATE_STOP = 0.01         # predicted collision probability below which a decided slot stops checking
SURROGATE_ROUNDS = 3
QUEUE_STEPS = 4               # timed steps whose inflations the queued form runs in one call
CPU_SAMPLE_SCENES = (0, 1, 2, 3)
CPU_SAMPLE = ("scenes 0-3 of the workload (7-DOF, 14-DOF, 7-DOF, 14-DOF), each scene's first seed edge (found with "
              "the oracle's checker), one inflation per step in that order, cycled; the same inflations in the "
              "reference arm and in the GPU arm's cpu_baseline leg")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    return ap.parse_args()


def bench_config():
    """The workload's description, identical in both arms."""
    return {"workload": WORKLOAD, "slots_per_gpu": NUM_SLOTS, "eizo_options": dict(EIZO_KW),
            "face_capacity": FACE_CAPACITY, "l2": L2_RULE, "cpu_sample": CPU_SAMPLE}


def box_domain(scene):
    d = scene.dim
    A = np.zeros((2 * d, d), np.float32)
    for i in range(d):
        A[2 * i, i], A[2 * i + 1, i] = -1, 1
    b = np.concatenate([[-scene.lower()[i], scene.upper()[i]] for i in range(d)]).astype(np.float32)
    return A, b


def scene_ranges(world: int):
    """Scene seeds of the fixed workload (world x 256 scenes, then spares) and
    each rank's contiguous [begin, end) range of equal predicted cost."""
    from csdecomp_b200 import scenes
    from csdecomp_b200.shard import cost_balanced_ranges
    n = NUM_SLOTS * world
    seeds = scenes.batch_scene_seeds(n + 128 * world, scenes.BATCH_SEED)
    costs = [scenes.batch_scene_cost(i, s) for i, s in enumerate(seeds[:n])]
    return seeds, cost_balanced_ranges(costs, world), n


def workload(begin: int, end: int, edges_per_scene: int, make_checkers, seeds, spare_begin: int):
    """Scenes [begin, end) of the workload with `edges_per_scene` free seed
    edges each. A scene in which 8 x 4096 uniform draws yield too few free seed
    edges is replaced by the next spare scene of the same plant family (spares
    from `spare_begin`; the number replaced is reported)."""
    from csdecomp_b200 import scenes
    out, skipped, spare = [], 0, spare_begin
    for i in range(begin, end):
        idx = i
        while True:
            sc = scenes.batch_scene(idx, seeds[idx])
            cp, ce = make_checkers(sc)
            e = scenes.seed_edges(sc, edges_per_scene, SEED_EDGE_SEED + 101 * idx, cp, ce)
            if len(e) == edges_per_scene:
                break
            skipped += 1
            spare += (spare - i) % 2  # same parity as i: the same plant family
            idx, spare = spare, spare + 2
            if idx >= len(seeds):
                raise RuntimeError("spare scenes exhausted")
        out.append((sc, e))
    return out, skipped


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_checkers(nthreads: int):
    from oracle import oracle as O

    def make(sc):
        return (lambda q: O.check_points(sc.plant, q, O.RULE_GPU, nthreads=nthreads),
                lambda a, b: O.check_edges(sc.plant, a, b, nthreads=nthreads)[0])
    return make


def cpu_sample_items(nthreads: int):
    """The CPU sample: (scene, (q0, q1)) for scenes CPU_SAMPLE_SCENES with
    their first seed edge, found with the oracle's checker (the same inputs
    in both arms)."""
    from csdecomp_b200 import scenes
    seeds = scenes.batch_scene_seeds(max(CPU_SAMPLE_SCENES) + 1, scenes.BATCH_SEED)
    make = oracle_checkers(nthreads)
    out = []
    for i in CPU_SAMPLE_SCENES:
        sc = scenes.batch_scene(i, seeds[i])
        cp, ce = make(sc)
        e = scenes.seed_edges(sc, 1, SEED_EDGE_SEED + 101 * i, cp, ce)
        if not e:
            raise RuntimeError(f"CPU sample scene {i} has no free seed edge")
        out.append((sc, e[0]))
    return out


def cpu_inflate(sc, q0, q1, nthreads: int, **overrides):
    """One inflation by the oracle's restated executeEizo; returns seconds."""
    from csdecomp_b200.api import EizoOptions
    from oracle import oracle as O
    kw = dict(EIZO_KW)
    kw.update(overrides)
    A0, b0 = box_domain(sc)
    t0 = time.perf_counter()
    O.eizo(sc.plant, q0, q1, A0, b0, EizoOptions(**kw), sc.inspector.robot_geometry_ids, capacity=FACE_CAPACITY,
           nthreads=nthreads)
    return time.perf_counter() - t0


def run_reference(args, rank):
    """CPU arm: the oracle's EI-ZO (restating the reference's executeEizo) on
    all host threads, one inflation of the CPU sample per step (cycled).
    Warm-up steps run the first EI-ZO iteration of a sample inflation only (a
    CPU inflation takes seconds to minutes; there is nothing to tune)."""
    if rank != 0:
        return
    ncores = os.cpu_count() or 1
    items = cpu_sample_items(ncores)
    for s in range(args.warmup):
        sc, (q0, q1) = items[s % len(items)]
        cpu_inflate(sc, q0, q1, ncores, max_iterations=1)
    times = []
    for s in range(args.steps):
        sc, (q0, q1) = items[s % len(items)]
        times.append(cpu_inflate(sc, q0, q1, ncores))
    total = float(sum(times))
    rate = len(times) / total
    line = {"metric": METRIC, "value": rate, "unit": "regions/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": bench_config(),
            "form": "CPU oracle, one inflation per step",
            "per_inflation_s": times,
            "cpu_baseline": {"value": rate, "unit": "regions/s", "cores": ncores, "kind": "port",
                             "sample": CPU_SAMPLE + "; the reference's CPU path cannot be built here (Eigen, glpk "
                                                    "and Bazel absent), so oracle/ restates executeEizo (OpenMP "
                                                    "over samples, all host threads)"},
            "e2e": {"value": rate, "unit": "regions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def time_device(torch, launch, reps: int, flush=None):
    """Mean device time (s) of `launch` over `reps` launches after 3 warm-up
    launches, CUDA events on the current stream, L2 flushed before each."""
    st = torch.cuda.current_stream()
    for _ in range(3):
        launch()
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.fill_(1)
        e0, e1 = _events(torch)
        e0.record(st)
        launch()
        e1.record(st)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3)
    return float(np.mean(ts))


def roofline_point_check(csd, scene, torch, dev, flush):
    """Fused FK + pair sweep on collision-free configurations of the 7-DOF /
    200-primitive scene: every pair is evaluated, so the FLOP count is exact."""
    from csdecomp_b200 import _capi as C
    import ctypes
    h = csd.plant_handle(scene.plant)
    fl = h.flops()
    q = scene.random_configs(200000, 77)
    free = q[csd.CheckCollisionFreeCuda(q.T, scene.plant) == 1]
    h.set_culling(False)  # the full sweep that the FLOP count describes
    n = 1 << 20
    reps = int(np.ceil(n / len(free)))
    qf = np.ascontiguousarray(np.tile(free, (reps, 1))[:n])
    tq = torch.from_numpy(qf).to(dev)
    out = torch.zeros(n, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream()

    def launch():
        C.check(C.lib().csd_check_points(h.handle, C.ptr(tq.data_ptr()), ctypes.c_int64(n), None, 0,
                                         ctypes.c_float(0), None, 0, C.ptr(out.data_ptr()), C.CSD_PTR_DEVICE,
                                         ctypes.c_void_p(st.cuda_stream)))
    t = time_device(torch, launch, 5, flush)
    assert int(out.sum().item()) == n, "roofline configurations must all be free"
    h.set_culling(True)
    t_culled = time_device(torch, launch, 3, flush)
    flops = fl["total"] * n
    fma_flops, fma_s = ctypes.c_double(), ctypes.c_double()
    C.check(C.lib().csd_fp32_fma_probe(ctypes.c_int64(20000), ctypes.byref(fma_flops), ctypes.byref(fma_s)))
    peak = fma_flops.value / fma_s.value
    achieved = flops / t
    return {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": CHECKER_TRAFFIC_BYTES,
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of this launch, one ncu capture "
                              "(profiles/check_points_kernel_1M_full_sweep.md)",
            "kernel": "check_points_kernel (fused FK + pair sweep; the batched check stage runs the same device code), "
                      "link-level broad phase off",
            "launch_ms_with_broad_phase": t_culled * 1e3,
            "per_config_flop": fl, "configs_per_launch": n, "launch_ms": t * 1e3,
            "peak_source": "measured FP32 FMA probe (csd_fp32_fma_probe) in this run",
            "workload": "1,048,576 collision-free configurations of the 7-DOF arm (80 spheres + 4 capsules) in "
                        "200 world primitives (full sweep, no early exit); L2 flushed between launches"}


# DRAM bytes per launch from ncu captures (profiles/): the full-sweep checker
# launch (2^20 configurations) and the sampler's launches of one 256-slot step.
CHECKER_TRAFFIC_BYTES = 29.5e6
SAMPLER_TRAFFIC_BYTES_PER_STEP = 216.4e6   # 147 launches, 156.5 MB read + 60.0 MB written


def check_workloads(csd, torch, dev, flush, cpu: bool):
    """Configs 1 and 2 (and the 0.8 m keep-out variant of config 2): device
    throughput with inputs resident (CUDA events), end to end through the
    host API (host arrays in and out), and, on rank 0 at N = 1, the oracle's
    restated CPU checks (collision_checker.cpp:9-53: CPU contact rule, early
    exit per configuration and per edge) on 1 thread and on all threads."""
    import ctypes
    from csdecomp_b200 import _capi as C
    from csdecomp_b200 import scenes
    from oracle import oracle as O
    st = torch.cuda.current_stream()
    ncores = os.cpu_count() or 1
    res = {}

    # config 1: point checks (+ transforms), 10^4 configurations, and the 10^6 sweep
    sc = scenes.point_check_scene()
    h = csd.plant_handle(sc.plant)
    c1 = {"scene": sc.description, "collision_pairs": int(sc.plant.num_collision_pairs),
          "full_sweep_flop_per_config": h.flops()["total"]}
    for n in (10_000, 1_000_000):
        q = sc.random_configs(n, 11 + n)
        tq = torch.from_numpy(q).to(dev)
        out = torch.zeros(n, dtype=torch.uint8, device=dev)
        tf = torch.zeros((n, h.num_links, 16), dtype=torch.float32, device=dev)

        def chk():
            C.check(C.lib().csd_check_points(h.handle, C.ptr(tq.data_ptr()), ctypes.c_int64(n), None, 0,
                                             ctypes.c_float(0), None, 0, C.ptr(out.data_ptr()), C.CSD_PTR_DEVICE,
                                             ctypes.c_void_p(st.cuda_stream)))

        def fk():
            C.check(C.lib().csd_fk(h.handle, C.ptr(tq.data_ptr()), ctypes.c_int64(n), C.ptr(tf.data_ptr()),
                                   C.CSD_PTR_DEVICE, ctypes.c_void_p(st.cuda_stream)))
        reps = 50 if n <= 10_000 else 10
        t_chk = time_device(torch, chk, reps, flush)
        t_fk = time_device(torch, fk, reps, flush)
        free = out.cpu().numpy()
        t0 = time.perf_counter()
        for _ in range(5):
            csd.CheckCollisionFreeCuda(q.T, sc.plant)
        t_e2e = (time.perf_counter() - t0) / 5
        e = {"configs": n, "configs_per_s": n / t_chk, "check_ms": t_chk * 1e3,
             "with_transforms_configs_per_s": n / (t_chk + t_fk), "fk_ms": t_fk * 1e3,
             "free_fraction": float(free.mean()), "e2e_configs_per_s": n / t_e2e}
        if n == 10_000:
            _, sd = O.signed_distance(sc.plant, q, nthreads=ncores)
            e["band_configs"] = int((np.abs(sd) <= 1e-5).sum())
            ref = O.check_points(sc.plant, q, O.RULE_GPU, nthreads=ncores)
            outside = np.abs(sd) > 1e-5
            e["verdicts_equal_oracle_outside_band"] = bool((free[outside] == ref[outside]).all())
            if cpu:
                t1 = time.perf_counter()
                O.check_points(sc.plant, q, O.RULE_CPU, nthreads=1)
                s1 = time.perf_counter() - t1
                t1 = time.perf_counter()
                O.check_points(sc.plant, q, O.RULE_CPU, nthreads=ncores)
                sa = time.perf_counter() - t1
                e["cpu"] = {"configs_per_s_1_thread": n / s1, "configs_per_s_all_threads": n / sa,
                            "threads": ncores, "kind": "port (oracle checkCollisionFree restatement, CPU rule)"}
        c1[f"n{n}"] = e
    res["config1_point_check"] = c1

    # config 2: edges, 10^5 segments, reference (L2) discretisation, early exit
    c2 = {}
    for label, ko in (("as_written", 0.0), ("keepout_0.8m", 0.8)):
        sc = scenes.edge_check_scene(keepout=ko)
        h = csd.plant_handle(sc.plant)
        n = 100_000
        s = sc.random_configs(n, 21)
        e_ = sc.random_configs(n, 22)
        ts, te = torch.from_numpy(s).to(dev), torch.from_numpy(e_).to(dev)
        out = torch.zeros(n, dtype=torch.uint8, device=dev)
        pts = torch.zeros(n, dtype=torch.int64, device=dev)

        def edges():
            C.check(C.lib().csd_check_edges(h.handle, C.ptr(ts.data_ptr()), C.ptr(te.data_ptr()), ctypes.c_int64(n),
                                            ctypes.c_float(0.01), C.CSD_EDGE_L2_REF, C.ptr(out.data_ptr()),
                                            C.ptr(pts.data_ptr()), C.CSD_PTR_DEVICE, ctypes.c_void_p(st.cuda_stream)))
        t_e = time_device(torch, edges, 10, flush)
        t0 = time.perf_counter()
        for _ in range(3):
            csd.CheckEdgesCollisionFreeCuda(s.T, e_.T, sc.plant)
        t_e2e = (time.perf_counter() - t0) / 3
        p = pts.cpu().numpy()
        ent = {"segments": n, "scene": sc.description + (f", {ko} m keep-out" if ko else ""),
               "edges_per_s": n / t_e, "check_ms": t_e * 1e3, "points_checked_per_s": float(p.sum()) / t_e,
               "mean_points_checked": float(p.mean()), "free_fraction": float(out.float().mean().item()),
               "e2e_edges_per_s": n / t_e2e}
        if cpu:
            m_all = n if ko == 0.0 else 2_000
            m_one = n // 10 if ko == 0.0 else 200
            t1 = time.perf_counter()
            O.check_edges(sc.plant, s[:m_one], e_[:m_one], 0.01, O.EDGE_L2_REF, O.RULE_CPU, nthreads=1)
            s1 = time.perf_counter() - t1
            t1 = time.perf_counter()
            O.check_edges(sc.plant, s[:m_all], e_[:m_all], 0.01, O.EDGE_L2_REF, O.RULE_CPU, nthreads=ncores)
            sa = time.perf_counter() - t1
            ent["cpu"] = {"edges_per_s_1_thread": m_one / s1, "edges_per_s_all_threads": m_all / sa,
                          "threads": ncores, "sample_edges": {"1_thread": m_one, "all_threads": m_all},
                          "kind": "port (oracle checkEdgeCollisionFree restatement, CPU rule)"}
        c2[label] = ent
    res["config2_edge_check"] = c2
    return res


def single_inflations(csd, torch, cpu: bool):
    """Config 3: plain GPU EI-ZO (one CudaEdgeInflator.inflateEdge per region)
    on 20 seed edges of length U[0.1, 0.5] rad of the 7-DOF / 200-primitive
    arm (0.8 m keep-out), events around each call; the oracle's EI-ZO on two
    of them on all host threads."""
    from csdecomp_b200 import scenes
    sc = scenes.edge_check_scene(keepout=0.8)

    def gpu_checkers(s):
        return (lambda q: csd.CheckCollisionFreeCuda(q.T, s.plant),
                lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, s.plant))
    cp, ce = gpu_checkers(sc)
    edges = scenes.seed_edges(sc, 20, 33, cp, ce, length=(0.1, 0.5))
    dom = csd.HPolyhedron()
    dom.MakeBox(sc.lower(), sc.upper())
    opt = csd.EizoOptions(**EIZO_KW)
    inf = csd.CudaEdgeInflator(sc.plant, sc.inspector.robot_geometry_ids, opt, dom, face_capacity=FACE_CAPACITY)
    inf.inflateEdge(edges[0][0], edges[0][1], None, 0.0, verbose=False)  # warm-up
    st = torch.cuda.current_stream()
    total, faces, iters = 0.0, [], []
    for q0, q1 in edges:
        e0, e1 = _events(torch)
        e0.record(st)
        P = inf.inflateEdge(q0, q1, None, 0.0, verbose=False)
        e1.record(st)
        e1.synchronize()
        total += e0.elapsed_time(e1) * 1e-3
        faces.append(P.A().shape[0])
        iters.append(len(inf.last_info.iteration_info))
    out = {"scene": sc.description + ", 0.8 m keep-out", "inflations": len(edges),
           "regions_per_s": len(edges) / total, "mean_faces": float(np.mean(faces)),
           "mean_iterations": float(np.mean(iters))}
    if cpu:
        ncores = os.cpu_count() or 1
        ts = [cpu_inflate(sc, q0, q1, ncores) for q0, q1 in edges[:2]]
        out["cpu"] = {"regions_per_s": 2 / sum(ts), "per_inflation_s": ts, "threads": ncores, "kind": "port",
                      "sample": "the first two of the 20 seed edges"}
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.warmup < 1:
        raise SystemExit("--warmup must be >= 1")
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    from csdecomp_b200.shard import reduce_timing

    def gpu_checkers(sc):
        return (lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant))

    steps_total = args.warmup + args.steps
    seeds, ranges, n_global = scene_ranges(world)
    begin, end = ranges[rank]
    items, skipped = workload(begin, end, steps_total, gpu_checkers, seeds, n_global + 128 * rank)
    nslots = len(items)
    scs = [sc for sc, _ in items]
    doms = []
    for sc in scs:
        d = csd.HPolyhedron()
        d.MakeBox(sc.lower(), sc.upper())
        doms.append(d)
    opt = csd.EizoOptions(**EIZO_KW)
    slot_plant = list(range(nslots))

    def step_inputs(s):
        return [e[s][0] for _, e in items], [e[s][1] for _, e in items]

    # surrogate: one net per scene, trained on configurations labelled by the exact checker
    from csdecomp_b200.surrogate import CollisionSurrogate, training_set
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    xs, ys = [], []
    for i, (sc, e) in enumerate(items):
        x, y = training_set(sc, e, SURROGATE_ROWS, seed=SURROGATE_SEED + begin + i)
        xs.append(x)
        ys.append(y)
    t_label = time.perf_counter() - t0
    bank = CollisionSurrogate([sc.dim for sc in scs], seed=SURROGATE_SEED)
    t0 = time.perf_counter()
    hist = bank.train(xs, ys, batch=512, epochs=SURROGATE_EPOCHS, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    pos = float(np.mean([y.mean() for y in ys]))

    def timed_run(batch, nvtx=False):
        """W warm-up steps (the first autotunes), then the K timed steps (in
        the NVTX range "timed" when asked)."""
        for s in range(args.warmup):
            q0s, q1s = step_inputs(s)
            batch.inflate(slot_plant, q0s, q1s, doms)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        if nvtx:
            torch.cuda.nvtx.range_push("timed")
        r = dict(dev_s=0.0, wall_s=0.0, configs=0, launches=0, faces=[], iters=[], h2d=0, d2h=0, first=None,
                 kept=[], step_s=[])
        for s in range(args.warmup, steps_total):
            q0s, q1s = step_inputs(s)
            flush.fill_(1)  # L2 flush between steps (outside the timed window)
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            regions = batch.inflate(slot_plant, q0s, q1s, doms)
            r["wall_s"] += time.perf_counter() - w0
            r["dev_s"] += batch.last_device_ms * 1e-3
            if r["first"] is None:
                r["first"] = regions
            if len(r["kept"]) < QUEUE_STEPS:
                r["kept"].append(regions)
            r["step_s"].append(batch.last_device_ms * 1e-3)
            r["configs"] += int(batch.last_configs_checked.sum())
            r["launches"] += batch.last_kernel_launches
            r["faces"] += [p.A().shape[0] for p in regions]
            r["iters"] += [int(x) for x in batch.last_iterations]
            r["h2d"] += sum(sc.dim * 8 + d.A().nbytes + d.b().nbytes for sc, d in zip(scs, doms)) + 8 * nslots + 4
            r["d2h"] += sum(p.A().nbytes + p.b().nbytes for p in regions) + 16 * int(batch.last_iterations.max()) \
                + 152 * nslots
        torch.cuda.synchronize()
        if nvtx:
            torch.cuda.nvtx.range_pop()
        return r

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    batched = csd.BatchedEdgeInflator([sc.plant for sc in scs], opt, max_slots=nslots, face_capacity=FACE_CAPACITY)
    rb = timed_run(batched)
    tuned_plain = batched.tuning()
    surrogate_batch = csd.BatchedEdgeInflator([sc.plant for sc in scs], opt, max_slots=nslots,
                                              face_capacity=FACE_CAPACITY)
    surrogate_batch.set_surrogate(bank, SURROGATE_STOP)
    with ClockSampler(local) as clk:
        rs = timed_run(surrogate_batch, nvtx=True)
    tuned_surr = surrogate_batch.tuning()
    first_regions = rb["first"]
    # roofline of the dominant kernel (the sampler): one profiled pass of the first timed step
    batched.set_profiling(True)
    q0s, q1s = step_inputs(args.warmup)
    batched.inflate(slot_plant, q0s, q1s, doms)
    stages = batched.stage_ms()
    s_ms = stages["sample"]
    s_flop = batched.sample_flops()
    batched.set_profiling(False)
    sampler_roofline = {"bound": "fp32", "achieved": s_flop / (s_ms * 1e-3) / 1e12, "peak": None, "unit": "TFLOP/s",
                        "frac": None, "traffic": SAMPLER_TRAFFIC_BYTES_PER_STEP,
                        "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum summed over the sampler "
                                          "launches of one timed step, one ncu capture "
                                          "(profiles/batch_sample_kernel_dram_traffic_one_step.md); step basis, "
                                          "as achieved",
                        "kernel": "batch_sample_kernel (hit-and-run, G lanes per chain, faces staged in shared memory; "
                                  "autotuned variant " + tuned_plain["sample_variant"] + "; regions beyond its "
                                  "staging: " + tuned_plain["large_region_variant"] + ")",
                        "flop_per_unit": batched.SAMPLE_FLOP_RULE,
                        "flop_per_step": s_flop, "kernel_ms_per_step": s_ms,
                        "share_of_step": s_ms / sum(stages.values()), "stage_ms": stages,
                        "timing": "CUDA events around every sampler launch of one profiled pass over the first timed "
                                  "step (stages launched one by one, same inputs and shapes as the graph)"}
    # plain GPU form (one CudaEdgeInflator call per region) on the first timed step's inputs
    plain_s, identical = 0.0, True
    st = torch.cuda.current_stream()
    q0s, q1s = step_inputs(args.warmup)
    for i, sc in enumerate(scs):
        inf = csd.CudaEdgeInflator(sc.plant, sc.inspector.robot_geometry_ids, opt, doms[i],
                                   face_capacity=FACE_CAPACITY)
        torch.cuda.synchronize()
        e0, e1 = _events(torch)
        e0.record(st)
        P = inf.inflateEdge(q0s[i], q1s[i], None, 0.0, verbose=False)
        e1.record(st)
        e1.synchronize()
        plain_s += e0.elapsed_time(e1) * 1e-3
        identical &= bool(np.array_equal(P.A(), first_regions[i].A()) and np.array_equal(P.b(), first_regions[i].b()))
        del inf
    # queued form: the inflations of the first QUEUE_STEPS timed steps in one call on the same slots (each
    # later inflation starts in the first slot that frees up), against those steps one call each
    qsteps = len(rb["kept"])
    qi0, qi1, qdom, qplant = [], [], [], []
    for j in range(qsteps):
        a0, a1 = step_inputs(args.warmup + j)
        qi0 += a0
        qi1 += a1
        qdom += doms
        qplant += slot_plant
    flush.fill_(1)
    torch.cuda.synchronize()
    qregions = batched.inflate(qplant, qi0, qi1, qdom)
    queued_s = batched.last_device_ms * 1e-3
    per_call_s = float(sum(rb["step_s"][:qsteps]))
    q_identical = all(np.array_equal(P.A(), R.A()) and np.array_equal(P.b(), R.b())
                      for P, R in zip(qregions, [x for regs in rb["kept"] for x in regs]))
    if dist:
        dev_s, wall_s, configs_all = reduce_timing(dist, dev, rs["dev_s"], rs["wall_s"], float(rs["configs"]))
        b_dev, _, b_cfg = reduce_timing(dist, dev, rb["dev_s"], rb["wall_s"], float(rb["configs"]))
        plain_s, _, regions_step = reduce_timing(dist, dev, plain_s, 0.0, float(nslots))
        queued_s, _, _ = reduce_timing(dist, dev, queued_s, 0.0, 0.0)
        per_call_s, _, _ = reduce_timing(dist, dev, per_call_s, 0.0, 0.0)
        idn = torch.tensor([1.0 if identical else 0.0], device=dev)
        dist.all_reduce(idn, op=dist.ReduceOp.MIN)
        identical = bool(idn.item() == 1.0)
    else:
        dev_s, wall_s, configs_all = rs["dev_s"], rs["wall_s"], float(rs["configs"])
        b_dev, b_cfg = rb["dev_s"], float(rb["configs"])
        regions_step = float(nslots)
    regions_all = regions_step * args.steps
    if rank == 0:
        value = regions_all / dev_s
        batched_value = regions_all / b_dev
        plain = regions_step / plain_s
        faces = np.asarray(rs["faces"])
        line = {"metric": METRIC, "value": value, "unit": "regions/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (checks), bf16 (surrogate MLP)",
                "data": "synthetic (seeded)",
                "config": bench_config(),
                "form": "surrogate + batched (BatchedEdgeInflator with a trained CollisionSurrogate, one slot per "
                        "scene, CUDA graph)",
                "parallelism": f"{world} independent ranks, contiguous scene ranges of equal predicted cost "
                               f"(rank 0: scenes {begin}..{end - 1})",
                "scenes_replaced": skipped,
                "surrogate": {"nets": len(scs), "architecture": "in->256->256->256->1 BF16, FP32 accumulate",
                              "training_rows": SURROGATE_ROWS * len(scs), "colliding_fraction": pos,
                              "epochs": SURROGATE_EPOCHS, "label_s": t_label, "train_s": t_train,
                              "final_loss": float(hist[-20:].mean()), "first_loss": float(hist[:20].mean()),
                              "stop_probability": SURROGATE_STOP,
                              "note": "trained once before the timed steps; every verdict is the exact "
                                      "checker's, admissibility uses the unchanged first-M test"},
                "autotuned": {"batched": tuned_plain["sample_variant"] + f", check cap {tuned_plain['check_item_cap']}",
                              "batched_large_regions": tuned_plain["large_region_variant"],
                              "surrogate": tuned_surr["sample_variant"],
                              "surrogate_large_regions": tuned_surr["large_region_variant"]},
                "configs_per_s": configs_all / dev_s,
                "configs_checked_per_step": configs_all / args.steps,
                "batched_gpu": {"value": batched_value, "unit": "regions/s", "configs_per_s": b_cfg / b_dev,
                                "configs_checked_per_step": b_cfg / args.steps,
                                "note": "same steps without the surrogate; regions identical to the plain form"},
                "plain_gpu": {"value": plain, "unit": "regions/s",
                              "sample": "the first timed step's inflations, one CudaEdgeInflator.inflateEdge "
                                        "call each", "identical_to_batched": identical},
                "queued_gpu": {"value": regions_step * qsteps / queued_s, "unit": "regions/s",
                               "same_inflations_one_call_per_step": regions_step * qsteps / per_call_s,
                               "inflations": int(regions_step * qsteps), "slots_per_gpu": nslots,
                               "identical_to_batched": q_identical,
                               "form": f"the inflations of the first {qsteps} timed steps in one BatchedEdgeInflator "
                                       "call on the same slots (each later inflation starts in the first slot that "
                                       "frees up), against the same steps one call each (batched form)"},
                "surrogate_batched_over_plain": value / plain,
                "batched_over_plain": batched_value / plain,
                "faces": {"mean": float(faces.mean()), "p50": float(np.median(faces)),
                          "p95": float(np.percentile(faces, 95)), "max": int(faces.max()), "min": int(faces.min()),
                          "share_over_300": float((faces > 300).mean()),
                          "note": "regions run to admissibility with capacity 4000; the workload's nominal "
                                  "'up to 300 hyperplanes' is exceeded by the share given (rank 0)"},
                "iterations": {"mean": float(np.mean(rs["iters"])), "max": int(np.max(rs["iters"]))},
                "e2e": {"value": regions_all / wall_s, "unit": "regions/s",
                        "h2d_bytes_per_step": rs["h2d"] // args.steps, "d2h_bytes_per_step": rs["d2h"] // args.steps,
                        "path": "BatchedEdgeInflator.inflate (surrogate set) with host numpy segments and polytopes "
                                "in, host polytopes out"},
                "gpu_launches": rs["launches"],
                "clocks": clk.summary()}
        line["roofline_checker"] = roofline_point_check(csd, scenes.edge_check_scene(keepout=0.8), torch, dev, flush)
        sampler_roofline["peak"] = line["roofline_checker"]["peak"]
        sampler_roofline["frac"] = sampler_roofline["achieved"] / sampler_roofline["peak"]
        sampler_roofline["peak_source"] = line["roofline_checker"]["peak_source"]
        line["roofline"] = sampler_roofline
        cpu = world == 1
        line["configs_1_2"] = check_workloads(csd, torch, dev, flush, cpu)
        line["config3_single_inflation"] = single_inflations(csd, torch, cpu)
        if cpu:
            ncores = os.cpu_count() or 1
            sample = cpu_sample_items(ncores)
            ts = [cpu_inflate(sc, q0, q1, ncores) for sc, (q0, q1) in sample]
            gpu_ts = []
            for sc, (q0, q1) in sample:
                dm = csd.HPolyhedron()
                dm.MakeBox(sc.lower(), sc.upper())
                inf = csd.CudaEdgeInflator(sc.plant, sc.inspector.robot_geometry_ids, opt, dm,
                                           face_capacity=FACE_CAPACITY)
                inf.inflateEdge(q0, q1, None, 0.0, verbose=False)  # warm-up
                e0, e1 = _events(torch)
                e0.record(st)
                inf.inflateEdge(q0, q1, None, 0.0, verbose=False)
                e1.record(st)
                e1.synchronize()
                gpu_ts.append(e0.elapsed_time(e1) * 1e-3)
            rate = len(ts) / sum(ts)
            line["cpu_baseline"] = {"value": rate, "unit": "regions/s", "cores": ncores, "kind": "port",
                                    "sample": CPU_SAMPLE + "; oracle's restated executeEizo with OpenMP",
                                    "per_inflation_s": ts,
                                    "gpu_plain_same_sample": {"regions_per_s": len(gpu_ts) / sum(gpu_ts),
                                                              "per_inflation_s": gpu_ts},
                                    "matched_ratio_plain_gpu_over_cpu": sum(ts) / sum(gpu_ts)}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
