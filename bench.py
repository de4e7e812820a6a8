#!/usr/bin/env python
"""Benchmark: EI-ZO regions/s on one B200 (plain GPU form) on the synthetic
7-DOF / 200-primitive scene, with the fused collision kernel's FP32 roofline
and the CPU oracle's EI-ZO on the host cores beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]

One step = one EI-ZO inflation (CudaEdgeInflator.inflateEdge) of a distinct
seed edge. N > 1 (torchrun): every rank inflates its own seed edges (weak
scaling, no collective on the data path); rank 0 prints one JSON line.
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
WORKLOAD = ("single EI-ZO inflation, plain GPU form: 7-DOF arm (80 spheres + 4 capsules), 200 world primitives "
            "(100 boxes + 100 spheres, centres U[-1,1]^3, 0.8 m base keep-out), seed edges U[0.1,0.5] rad, "
            "2000 particles, mixing 50, 9 bisection steps, <=10 faces/iteration, eps=0.01, delta=0.05, tau=0.5")
EIZO_KW = dict(num_particles=2000, mixing_steps=50, bisection_steps=9, max_hyperplanes_per_iteration=10,
               epsilon=0.01, delta=0.05, tau=0.5, max_iterations=500, configuration_margin=0.01, seed=1337)
SEED_EDGE_SEED = 3000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    return ap.parse_args()


def seed_edges(scene, count: int, check_points, check_edge):
    """Seeded pool of free seed edges: a free q0, a direction uniform on the
    sphere, length U[0.1, 0.5] rad, accepted iff the edge lies in the joint
    limits and is collision free (the reference's edge rule)."""
    rng = np.random.default_rng(SEED_EDGE_SEED)
    lo, hi = scene.lower(), scene.upper()
    out = []
    while len(out) < count:
        q = scene.random_configs(4096, int(rng.integers(1 << 30)))
        free = q[check_points(q) == 1]
        for q0 in free:
            d = rng.normal(size=q0.size)
            d /= np.linalg.norm(d)
            q1 = (q0 + rng.uniform(0.1, 0.5) * d).astype(np.float32)
            if np.all(q1 > lo) and np.all(q1 < hi) and check_edge(q0, q1):
                out.append((q0.copy(), q1))
                if len(out) == count:
                    break
    return out


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


def cpu_eizo_baseline(scene, edges, nthreads: int):
    from csdecomp_b200.api import EizoOptions
    from oracle import oracle as O
    d = scene.dim
    A0 = np.zeros((2 * d, d), np.float32)
    for i in range(d):
        A0[2 * i, i], A0[2 * i + 1, i] = -1, 1
    b0 = np.concatenate([[-scene.lower()[i], scene.upper()[i]] for i in range(d)]).astype(np.float32)
    opt = EizoOptions(**EIZO_KW)
    t0 = time.perf_counter()
    n = 0
    for q0, q1 in edges:
        O.eizo(scene.plant, q0, q1, A0, b0, opt, scene.inspector.robot_geometry_ids, nthreads=nthreads)
        n += 1
        if time.perf_counter() - t0 > 20.0:
            break
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args, rank):
    if rank != 0:
        return
    from csdecomp_b200 import scenes
    from oracle import oracle as O
    scene = scenes.edge_check_scene(keepout=0.8)
    ncores = os.cpu_count() or 1
    edges = seed_edges(scene, args.warmup + args.steps,
                       lambda q: O.check_points(scene.plant, q, O.RULE_GPU, nthreads=ncores),
                       lambda a, b: bool(O.check_edges(scene.plant, a[None], b[None], nthreads=ncores)[0][0]))
    d = scene.dim
    A0 = np.zeros((2 * d, d), np.float32)
    for i in range(d):
        A0[2 * i, i], A0[2 * i + 1, i] = -1, 1
    b0 = np.concatenate([[-scene.lower()[i], scene.upper()[i]] for i in range(d)]).astype(np.float32)
    from csdecomp_b200.api import EizoOptions
    opt = EizoOptions(**EIZO_KW)
    for q0, q1 in edges[:args.warmup]:
        O.eizo(scene.plant, q0, q1, A0, b0, opt, scene.inspector.robot_geometry_ids, nthreads=ncores)
    t0 = time.perf_counter()
    for q0, q1 in edges[args.warmup:]:
        O.eizo(scene.plant, q0, q1, A0, b0, opt, scene.inspector.robot_geometry_ids, nthreads=ncores)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": "regions/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": {"workload": WORKLOAD, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": v, "unit": "regions/s", "cores": ncores, "kind": "port",
                             "sample": f"{args.steps} inflations on all host threads (the reference's CPU path "
                                       "cannot be built here: Eigen/glpk/Bazel absent; oracle/ restates executeEizo)"},
            "e2e": {"value": v, "unit": "regions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def roofline_point_check(csd, scene, torch, dev):
    """Fused FK + pair sweep on collision-free configurations of the scene:
    every pair is evaluated, so the FLOP count is exact."""
    from csdecomp_b200 import _capi as C
    import ctypes
    h = csd.plant_handle(scene.plant)
    fl = h.flops()
    q = scene.random_configs(200000, 77)
    free = q[csd.CheckCollisionFreeCuda(q.T, scene.plant) == 1]
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
    for _ in range(2):
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
    t = float(np.mean(times))
    flops = fl["total"] * n
    fma_flops, fma_s = ctypes.c_double(), ctypes.c_double()
    C.check(C.lib().csd_fp32_fma_probe(ctypes.c_int64(20000), ctypes.byref(fma_flops), ctypes.byref(fma_s)))
    peak = fma_flops.value / fma_s.value
    achieved = flops / t
    return {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": None,
            "kernel": "check_points_kernel (fused FK + pair sweep)",
            "per_config_flop": fl, "configs_per_launch": n, "launch_ms": t * 1e3,
            "peak_source": "measured FP32 FMA probe (csd_fp32_fma_probe) in this run",
            "workload": "1,048,576 collision-free configurations of the bench scene (full sweep, no early exit); "
                        "L2 flushed between launches"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import csdecomp_b200 as csd
    from csdecomp_b200 import scenes

    scene = scenes.edge_check_scene(keepout=0.8)
    total_edges = (args.warmup + args.steps) * world
    edges = seed_edges(scene, total_edges, lambda q: csd.CheckCollisionFreeCuda(q.T, scene.plant),
                       lambda a, b: csd.CheckEdgeCollisionFree(a, b, scene.plant))
    from csdecomp_b200.shard import reduce_timing, shard
    per_rank = args.warmup + args.steps
    mine = edges[rank * per_rank:(rank + 1) * per_rank]
    dom = csd.HPolyhedron()
    dom.MakeBox(scene.lower(), scene.upper())
    opt = csd.EizoOptions(**EIZO_KW)
    inf = csd.CudaEdgeInflator(scene.plant, scene.inspector.robot_geometry_ids, opt, dom)
    for q0, q1 in mine[:args.warmup]:
        inf.inflateEdge(q0, q1, None, 0.0, verbose=False)
    torch.cuda.synchronize()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    dev_s, wall_s, faces, configs, launches = 0.0, 0.0, 0, 0, 0
    d2h = 0
    with ClockSampler(local) as clk:
        for q0, q1 in mine[args.warmup:]:
            flush.fill_(1)  # L2 flush between steps (outside the timed window)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            w0 = time.perf_counter()
            e0.record(st)
            P = inf.inflateEdge(q0, q1, None, 0.0, verbose=False)
            e1.record(st)
            e1.synchronize()
            wall_s += time.perf_counter() - w0
            dev_s += e0.elapsed_time(e1) * 1e-3
            it = inf.last_info.iteration_info
            faces += P.A().shape[0]
            configs += sum(i.num_samples_drawn + i.num_collisions_updated * opt.bisection_steps for i in it)
            launches += sum(3 + (2 if i.num_collisions_updated else 0) for i in it)
            d2h += P.A().shape[0] * (scene.dim + 1) * 4 + 16 * (len(it) + 1) + 4
    torch.cuda.synchronize()
    if dist:
        dev_s, wall_s, configs_all = reduce_timing(dist, dev, dev_s, wall_s, float(configs))
        dist.barrier()
    else:
        configs_all = float(configs)
    regions = args.steps * world
    if rank == 0:
        value = regions / dev_s
        line = {"metric": METRIC, "value": value, "unit": "regions/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": {"workload": WORKLOAD, "form": "plain GPU (one inflation per call)",
                           "parallelism": f"{world} independent ranks",
                           "l2": "flushed between steps (256 MB write)"},
                "configs_per_s": configs_all / dev_s,
                "mean_faces": faces / args.steps,
                "e2e": {"value": regions / wall_s, "unit": "regions/s",
                        "h2d_bytes_per_step": 2 * scene.dim * 4, "d2h_bytes_per_step": d2h // args.steps,
                        "path": "CudaEdgeInflator.inflateEdge with host numpy segment and host polytope out"},
                "gpu_launches": launches,
                "clocks": clk.summary()}
        line["roofline"] = roofline_point_check(csd, scene, torch, dev)
        if world == 1:
            rate, n, dt = cpu_eizo_baseline(scene, mine[args.warmup:args.warmup + 4], os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": rate, "unit": "regions/s", "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": f"{n} inflations of the same seed edges ({dt:.1f} s) by the oracle's "
                                              "restated executeEizo with OpenMP"}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
