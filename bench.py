#!/usr/bin/env python
"""Benchmark: EI-ZO regions/s and configs/s on one B200, batched form: 256
inflations per step on 256 seeded scenes (7-DOF and 14-DOF plants mixed), the
plain GPU form (one inflation per call) on the same inputs beside it, the
collision kernel's FP32 roofline and the CPU oracle's EI-ZO on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]

One step = one BatchedEdgeInflator.inflate of 256 seed edges, one per scene.
N > 1 (torchrun): every rank inflates its own 256 scenes (weak scaling, no
collective on the data path); rank 0 prints one JSON line.
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
WORKLOAD = ("batched EI-ZO: 256 inflations per step, one per seeded scene (even: 7-DOF arm, 80 spheres + 4 "
            "capsules; odd: 14-DOF two-arm plant, 2 x (40 spheres + 2 capsules)); U{50..400} world primitives per "
            "scene (half boxes, half spheres, centres U[-1,1]^3, 0.8 m keep-out around each base); seed edges "
            "U[0.05,1.0] rad in free space; domain = joint-limit box; 2000 particles, mixing 50, 9 bisection steps, "
            "<=10 faces/iteration, eps=0.01, delta=0.05, tau=0.5")
SEED_EDGE_SEED = 3000
SURROGATE_ROWS = 16384        # labelled configurations per scene (4.2 M over the 256 scenes)
SURROGATE_EPOCHS = 6
SURROGATE_SEED = 5000
SURROGATE_STOP = 0.01         # predicted collision probability below which a decided slot stops checking
SURROGATE_ROUNDS = 3
RANK_SCENE_STRIDE = 7919


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    return ap.parse_args()


def box_domain(scene):
    d = scene.dim
    A = np.zeros((2 * d, d), np.float32)
    for i in range(d):
        A[2 * i, i], A[2 * i + 1, i] = -1, 1
    b = np.concatenate([[-scene.lower()[i], scene.upper()[i]] for i in range(d)]).astype(np.float32)
    return A, b


def workload(rank: int, count: int, edges_per_scene: int, make_checkers):
    """`count` scenes of the batched workload with `edges_per_scene` free seed
    edges each. Scenes come from the rank's seeded stream in order; a scene in
    which 8 x 4096 uniform draws yield too few free seed edges is skipped (the
    number skipped is reported)."""
    from csdecomp_b200 import scenes
    seeds = scenes.batch_scene_seeds(4 * count + 64, scenes.BATCH_SEED + RANK_SCENE_STRIDE * rank)
    out, skipped = [], 0
    for i, s in enumerate(seeds):
        sc = scenes.batch_scene(i, s)
        cp, ce = make_checkers(sc)
        e = scenes.seed_edges(sc, edges_per_scene, SEED_EDGE_SEED + 101 * i + rank, cp, ce)
        if len(e) < edges_per_scene:
            skipped += 1
            continue
        out.append((sc, e))
        if len(out) == count:
            return out, skipped
    raise RuntimeError("scene stream exhausted")


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


def cpu_eizo(items, nthreads: int, budget_s: float):
    """The oracle's restated executeEizo on (scene, edge) items until the time
    budget runs out; returns (regions/s, regions, seconds)."""
    from csdecomp_b200.api import EizoOptions
    from oracle import oracle as O
    opt = EizoOptions(**EIZO_KW)
    t0 = time.perf_counter()
    n = 0
    for sc, (q0, q1) in items:
        A0, b0 = box_domain(sc)
        O.eizo(sc.plant, q0, q1, A0, b0, opt, sc.inspector.robot_geometry_ids, capacity=FACE_CAPACITY,
               nthreads=nthreads)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args, rank):
    """CPU arm: the oracle's EI-ZO (restating the reference's executeEizo) on
    the host cores, one inflation per step, on the first W + K scenes of the
    same workload with their first timed seed edge. A CPU inflation takes tens
    of seconds, so warm-up stops after 30 s and the timed steps after 120 s;
    the line reports how many inflations ran."""
    if rank != 0:
        return
    ncores = os.cpu_count() or 1
    items, skipped = workload(0, args.warmup + args.steps, args.warmup + 1, oracle_checkers(ncores))
    items = [(sc, e[args.warmup]) for sc, e in items]
    cpu_eizo(items[:args.warmup], ncores, 30.0)
    rate, n, dt = cpu_eizo(items[args.warmup:], ncores, 120.0)
    line = {"metric": METRIC, "value": rate, "unit": "regions/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 * dt / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "form": "CPU, one inflation per step", "l2": "n/a (CPU)",
                       "scenes_skipped": skipped},
            "cpu_baseline": {"value": rate, "unit": "regions/s", "cores": ncores, "kind": "port",
                             "sample": f"{n} inflations (scenes {args.warmup}..{args.warmup + n - 1} of the "
                                       "workload, one seed edge each) on all host threads; the reference's CPU path "
                                       "cannot be built here (Eigen, glpk and Bazel absent), so oracle/ restates "
                                       "executeEizo"},
            "e2e": {"value": rate, "unit": "regions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def roofline_point_check(csd, scene, torch, dev):
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
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream()

    def launch():
        C.check(C.lib().csd_check_points(h.handle, C.ptr(tq.data_ptr()), ctypes.c_int64(n), None, 0,
                                         ctypes.c_float(0), None, 0, C.ptr(out.data_ptr()), C.CSD_PTR_DEVICE,
                                         ctypes.c_void_p(st.cuda_stream)))
    for _ in range(3):
        launch()
    times = []
    for _ in range(5):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        launch()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    assert int(out.sum().item()) == n, "roofline configurations must all be free"
    culled = []
    h.set_culling(True)
    for _ in range(3):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        launch()
        e1.record(st)
        e1.synchronize()
        culled.append(e0.elapsed_time(e1) * 1e-3)
    t = float(np.mean(times))
    flops = fl["total"] * n
    fma_flops, fma_s = ctypes.c_double(), ctypes.c_double()
    C.check(C.lib().csd_fp32_fma_probe(ctypes.c_int64(20000), ctypes.byref(fma_flops), ctypes.byref(fma_s)))
    peak = fma_flops.value / fma_s.value
    achieved = flops / t
    return {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": None,
            "kernel": "check_points_kernel (fused FK + pair sweep; the batched check stage runs the same device code), "
                      "link-level broad phase off",
            "launch_ms_with_broad_phase": float(np.mean(culled)) * 1e3,
            "per_config_flop": fl, "configs_per_launch": n, "launch_ms": t * 1e3,
            "peak_source": "measured FP32 FMA probe (csd_fp32_fma_probe) in this run",
            "workload": "1,048,576 collision-free configurations of the 7-DOF arm (80 spheres + 4 capsules) in "
                        "200 world primitives (full sweep, no early exit); L2 flushed between launches"}


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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes
    from csdecomp_b200.shard import reduce_timing

    def gpu_checkers(sc):
        return (lambda q: csd.CheckCollisionFreeCuda(q.T, sc.plant),
                lambda a, b: csd.CheckEdgesCollisionFreeCuda(a.T, b.T, sc.plant))

    steps_total = args.warmup + args.steps
    items, skipped = workload(rank, NUM_SLOTS, steps_total, gpu_checkers)
    scs = [sc for sc, _ in items]
    doms = []
    for sc in scs:
        d = csd.HPolyhedron()
        d.MakeBox(sc.lower(), sc.upper())
        doms.append(d)
    opt = csd.EizoOptions(**EIZO_KW)
    slot_plant = list(range(NUM_SLOTS))

    def step_inputs(s):
        return [e[s][0] for _, e in items], [e[s][1] for _, e in items]

    # surrogate: one net per scene, trained on configurations labelled by the exact checker
    from csdecomp_b200.surrogate import CollisionSurrogate, training_set
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    xs, ys = [], []
    for i, (sc, e) in enumerate(items):
        x, y = training_set(sc, e, SURROGATE_ROWS, seed=SURROGATE_SEED + i)
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
        r = dict(dev_s=0.0, wall_s=0.0, configs=0, launches=0, faces=[], iters=[], h2d=0, d2h=0, first=None)
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
            r["configs"] += int(batch.last_configs_checked.sum())
            n_graph = int(batch.last_iterations.max())
            r["launches"] += n_graph * (6 if batch_surrogate(batch) is None else 7 + 2 * SURROGATE_ROUNDS)
            r["faces"] += [p.A().shape[0] for p in regions]
            r["iters"] += [int(x) for x in batch.last_iterations]
            r["h2d"] += sum(sc.dim * 8 + d.A().nbytes + d.b().nbytes for sc, d in zip(scs, doms)) + 8 * NUM_SLOTS + 4
            r["d2h"] += sum(p.A().nbytes + p.b().nbytes for p in regions) + 16 * n_graph + 144 * NUM_SLOTS
        torch.cuda.synchronize()
        if nvtx:
            torch.cuda.nvtx.range_pop()
        return r

    def batch_surrogate(batch):
        return getattr(batch, "_surrogate", None)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    batched = csd.BatchedEdgeInflator([sc.plant for sc in scs], opt, max_slots=NUM_SLOTS, face_capacity=FACE_CAPACITY)
    rb = timed_run(batched)
    tuned_plain = batched.tuning()
    surrogate_batch = csd.BatchedEdgeInflator([sc.plant for sc in scs], opt, max_slots=NUM_SLOTS,
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
                        "frac": None, "traffic": None,
                        "kernel": "batch_sample_kernel (hit-and-run, G lanes per chain, faces staged in shared memory; "
                                  "autotuned variant " + tuned_plain["sample_variant"] + "; regions beyond its "
                                  "staging: " + tuned_plain["large_region_variant"] + ")",
                        "flop_per_unit": "4 d F per chain and mixing step (two length-d dot products per face, "
                                         "FMA = 2), summed over the slots and iterations of the step",
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
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        P = inf.inflateEdge(q0s[i], q1s[i], None, 0.0, verbose=False)
        e1.record(st)
        e1.synchronize()
        plain_s += e0.elapsed_time(e1) * 1e-3
        identical &= bool(np.array_equal(P.A(), first_regions[i].A()) and np.array_equal(P.b(), first_regions[i].b()))
        del inf
    if dist:
        dev_s, wall_s, configs_all = reduce_timing(dist, dev, rs["dev_s"], rs["wall_s"], float(rs["configs"]))
        b_dev, _, b_cfg = reduce_timing(dist, dev, rb["dev_s"], rb["wall_s"], float(rb["configs"]))
        plain_s, _, _ = reduce_timing(dist, dev, plain_s, 0.0, 0.0)
        dist.barrier()
    else:
        dev_s, wall_s, configs_all = rs["dev_s"], rs["wall_s"], float(rs["configs"])
        b_dev, b_cfg = rb["dev_s"], float(rb["configs"])
    regions_all = NUM_SLOTS * args.steps * world
    if rank == 0:
        value = regions_all / dev_s
        batched_value = regions_all / b_dev
        plain = NUM_SLOTS * world / plain_s
        line = {"metric": METRIC, "value": value, "unit": "regions/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 (checks), bf16 (surrogate MLP)",
                "data": "synthetic (seeded)",
                "config": {"workload": WORKLOAD,
                           "form": "surrogate + batched (BatchedEdgeInflator with a trained CollisionSurrogate, "
                                   "256 slots, CUDA graph)",
                           "parallelism": f"{world} independent ranks",
                           "l2": "flushed between steps (256 MB write)", "scenes_skipped": skipped,
                           "face_capacity": FACE_CAPACITY,
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
                                         "surrogate_large_regions": tuned_surr["large_region_variant"]}},
                "configs_per_s": configs_all / dev_s,
                "configs_checked_per_step": configs_all / args.steps / world,
                "batched_gpu": {"value": batched_value, "unit": "regions/s", "configs_per_s": b_cfg / b_dev,
                                "configs_checked_per_step": b_cfg / args.steps / world,
                                "note": "same steps without the surrogate; regions identical to the plain form"},
                "plain_gpu": {"value": plain, "unit": "regions/s",
                              "sample": "the first timed step's 256 inflations, one CudaEdgeInflator.inflateEdge "
                                        "call each", "identical_to_batched": identical},
                "surrogate_batched_over_plain": value / plain,
                "batched_over_plain": batched_value / plain,
                "faces": {"mean": float(np.mean(rs["faces"])), "max": int(np.max(rs["faces"])),
                          "min": int(np.min(rs["faces"]))},
                "iterations": {"mean": float(np.mean(rs["iters"])), "max": int(np.max(rs["iters"]))},
                "e2e": {"value": regions_all / wall_s, "unit": "regions/s",
                        "h2d_bytes_per_step": rs["h2d"] // args.steps, "d2h_bytes_per_step": rs["d2h"] // args.steps,
                        "path": "BatchedEdgeInflator.inflate (surrogate set) with host numpy segments and polytopes "
                                "in, host polytopes out"},
                "gpu_launches": rs["launches"],
                "clocks": clk.summary()}
        line["roofline_checker"] = roofline_point_check(csd, scenes.edge_check_scene(keepout=0.8), torch, dev)
        sampler_roofline["peak"] = line["roofline_checker"]["peak"]
        sampler_roofline["frac"] = sampler_roofline["achieved"] / sampler_roofline["peak"]
        sampler_roofline["peak_source"] = line["roofline_checker"]["peak_source"]
        line["roofline"] = sampler_roofline
        if world == 1:
            sample = [(sc, e[args.warmup]) for sc, e in items[:8]]
            rate, n, dt = cpu_eizo(sample, os.cpu_count() or 1, 20.0)
            line["cpu_baseline"] = {"value": rate, "unit": "regions/s", "cores": os.cpu_count() or 1,
                                    "kind": "port",
                                    "sample": f"{n} inflations of the first timed step's seed edges ({dt:.1f} s) by "
                                              "the oracle's restated executeEizo with OpenMP"}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
