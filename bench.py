#!/usr/bin/env python
"""Benchmark of the ATRBVH build-and-traverse path on B200.

Workload (the clustered-scene configuration): 4,194,304 fp32 triangles
(75% from 64 anisotropic Gaussians, 25% ground-plane quad grid), seed 0.
One step = LBVH (30-bit Morton, onesweep sort, fused Karras build + refit)
-> ATRBVH (treelet 9, 2 iterations) -> collapse (Ci 1.2, Ct 1.0) -> Compact2
flatten -> closest-hit traversal of 1920x1080 pinhole primary rays (eye
(0.5, 0.5, -1.5), 60 degree vertical field of view) -> one cosine-weighted
diffuse bounce per hit -> traversal of the bounces.

value = build throughput in Mtri/s (Morton through collapse, device-resident
input, CUDA events on the library's stream), summed over ranks; traversal
Mrays/s is reported beside it.  e2e repeats the build through the public C ABI
from pinned host vertices (H2D inside the timed region) to the SAH read back
on the host.  With --gpus N > 1 every rank builds its own replica (the path
has no data exchange for a single mesh).  After the K timed steps the default
line also carries: a sustained run of the same step (>= 1 s, with its own
clock record), the timed build's SAH against the oracle's committed value,
the 4096-mesh batched-vs-plain figures and serving p50/p99 at three arrival
rates, and the host-core baseline on the whole scene.

--impl reference times the checker's CPU restatement of the same pipeline on
all host cores, on the whole workload scene per step (the reference has no CPU
implementation of this path, and its CUDA build is not run); it loads nothing
from the product library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_TRIS = 4194304
WIDTH, HEIGHT = 1920, 1080
METRIC = "ATRBVH build Mtri/s at equal SAH, batched vs plain; Mrays/s; p99 latency"
WORKLOAD = ("clustered scene 4,194,304 tris (75% 64-Gaussian mixture, 25% 1024x512 ground-plane quads): "
            "LBVH 30-bit + ATRBVH(9,2) + collapse + Compact2, closest-hit trace of 1920x1080 primary "
            "rays + 1 diffuse bounce per hit")
# Algorithmic bytes per triangle (reference data types) per phase: Morton reads
# 48 B and writes key + index; each of the 4 sort passes reads and writes key +
# index after a 4-B histogram read; Karras build 40 B + refit 180 B; each ATRBVH
# iteration reads every node's parent/left/right/area/box once (48 B x 2 nodes),
# writes subtree count and nodesSah (8 B x 2) and a child record and counter per
# internal node (24 B).
BYTES_PER_TRI = {"morton": 56.0, "sort": 4.0 + 16.0 * 4, "build": 40.0 + 180.0, "atrbvh": 2 * 136.0}
REFIT_BYTES_PER_TRI = 180.0  # vertex gather 48, dataIndex 4, parents 8, boxes 64, areas 8, counters 8, siblings 32, children 8
# DRAM bytes per triangle of the ATRBVH phase (both iterations) from an ncu
# capture of this bench step at 2,097,152 triangles (dram__bytes_read.sum +
# dram__bytes_write.sum per step: k_levels_pp_hist 88.2 MB, k_level_hist 33.7,
# k_level_groups 1325.9 + 263.4 + 54.4, k_atrbvh 8.4), scaled by triangle count.
ATRBVH_DRAM_BYTES_PER_TRI = (88.2 + 33.7 + 1325.9 + 263.4 + 54.4 + 8.4) * 1e6 / 2097152


def _read_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return {"hbm_gbs": float(d["hbm_gbs"]), "src": "measured"}
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "src": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, interval_ms: int = 10):
        self.device = device
        self.interval_ms = interval_ms
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_pipeline(v: np.ndarray, threads: int) -> float:
    """Host-core LBVH + ATRBVH(9,2) + collapse on v; returns seconds."""
    import oracle as O
    t0 = time.perf_counter()
    mn, mx = O.scene_aabb(v)
    t, _, _ = O.build_lbvh(v, mn, mx, threads=threads)
    a = O.atrbvh(t, 9, 2, threads=threads)
    O.collapse(a)
    return time.perf_counter() - t0


def cpu_baseline(reps: int = 5) -> dict:
    """The host-core pipeline on the whole workload scene (generated by the
    checker's own generator), best of `reps` after one warm-up."""
    import oracle as O
    threads = O.max_threads()
    v = O.gen_scene(O.SCENE_CLUSTERED, N_TRIS, 0)
    cpu_pipeline(v, threads)  # warm-up
    secs = min(cpu_pipeline(v, threads) for _ in range(reps))
    return {"value": N_TRIS / secs / 1e6, "unit": "Mtri/s", "cores": threads, "kind": "port",
            "sample": f"the whole {N_TRIS}-triangle workload scene, LBVH+ATRBVH(9,2)+collapse, best of {reps} after "
                      f"1 warm-up"}


def golden_c2() -> dict | None:
    """Oracle SAH and digests of the clustered 4,194,304-triangle workload."""
    p = ROOT / "tests" / "golden" / "fullsize_oracle.json"
    if not p.exists():
        return None
    return json.loads(p.read_text()).get("c2")


def clustered_config(n_tris: int, world: int, rays_per_step: int) -> dict:
    """The workload description both arms print (identical for equal runs)."""
    return {"workload": WORKLOAD if n_tris == N_TRIS else f"{n_tris}-triangle instance of: {WORKLOAD}",
            "triangles": n_tris, "rays_per_step": int(rays_per_step), "treelet": 9, "iterations": 2,
            "morton_bits": 30, "collapse_max_leaf": 0, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (201 MB of vertices); no flush"}


def run_ours(args, world, rank, local):
    import torch
    import atrbvh_b200 as ab
    torch.cuda.set_device(local)
    ctx = ab.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    n_tris = args.triangles
    v = ab.gen_scene(ab.SCENE_CLUSTERED, n_tris, 0)
    scene = ab.SceneWrapper(ctx, v)  # scene box reduced on the device
    prim = ab.gen_rays_pinhole(WIDTH, HEIGHT)
    nr = len(prim)
    with torch.cuda.stream(stream):
        rays = torch.from_numpy(prim.reshape(-1)).to("cuda", non_blocking=False)
        res = torch.zeros(nr * 4, dtype=torch.int32, device="cuda")
        bounce = torch.zeros_like(rays)
        res2 = torch.zeros_like(res)
    torch.cuda.synchronize()

    # The steady-state step: the build plan (LBVH 30-bit -> ATRBVH(9,2) ->
    # collapse -> Compact2, one CUDA graph launch), then the primary trace, the
    # bounce generation and the bounce trace.
    plan = ab.BuildPlan(scene, optimizer=1, treelet=9, iterations=2, flatten=True)
    build_times: list[float] = []

    trace_events: list[tuple] = []

    def traces(bvh, record: bool = False):
        def timed(fn):
            if not record:
                fn()
                return
            ta = torch.cuda.Event(enable_timing=True)
            tb = torch.cuda.Event(enable_timing=True)
            ta.record(stream)
            fn()
            tb.record(stream)
            trace_events.append((ta, tb))
        timed(lambda: bvh.trace(rays.data_ptr(), nr, res.data_ptr()))
        ab.check(ab.lib().atr_gen_bounce_rays(ctx.handle, scene.handle, rays.data_ptr(), res.data_ptr(), nr, 1,
                                              bounce.data_ptr()))
        timed(lambda: bvh.trace(bounce.data_ptr(), nr, res2.data_ptr()))

    def step(record: bool = False):
        plan.run(graph=True)
        bvh = plan.compact()  # reads the layout's sizes: one small device-to-host copy
        if record:
            build_times.append(plan.times()[0])
        traces(bvh, record)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()

    # ---- device-resident timed region: exactly K steps ----
    # The plan's graph carries only its two build marks here; the per-phase
    # marks (an event node per stage boundary) are taken in a separate pass.
    clocks = ClockSampler(local)
    launches0 = ctx.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(record=True)
    ev1.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    launches = ctx.launch_count() - launches0
    total_ms = ev0.elapsed_time(ev1)
    trace_ms = sum(a.elapsed_time(b) for a, b in trace_events) / args.steps  # both trace launches
    rays_per_step = 2 * nr
    build_ms = statistics.mean(build_times)  # Morton through collapse, events inside the graph
    build_ms_max = max_over_ranks(build_ms, world)
    trace_ms_max = max_over_ranks(trace_ms, world)
    step_ms_max = max_over_ranks(total_ms / args.steps, world)

    # Per-phase device times: the same graph captured with phase marks, replayed
    # after the timed region (the marks' event nodes cost a few microseconds
    # each, so the timed build runs without them).
    ctx.set_timing(True)
    plan_phases: dict[str, float] = {}
    n_ph = max(3, min(20, args.steps))
    for i in range(n_ph + 1):  # the first replay captures the graph with its marks
        plan.run(graph=True)
        if i:
            for name, ms in plan.phase_times():
                plan_phases[name] = plan_phases.get(name, 0.0) + ms
    ctx.synchronize()
    ctx.set_timing(False)
    ph_ms = {k: x / n_ph for k, x in plan_phases.items()}
    ph_ms["trace"] = trace_ms  # both launches per step

    # ---- sustained: the same step repeated for at least a second, its own clock record ----
    sustained = None
    if args.sustain_s > 0:
        clocks2 = ClockSampler(local, interval_ms=50)
        barrier(world)
        torch.cuda.synchronize()
        clocks2.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < args.sustain_s or reps < 2:
            step()
            reps += 1
            if reps % 16 == 0:
                ctx.synchronize()
        e1.record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
        clk2 = clocks2.stop()
        s_ms = max_over_ranks(e0.elapsed_time(e1), world)
        sustained = {"steps": reps, "seconds": s_ms / 1e3, "ms_per_step": s_ms / reps,
                     "note": "whole steps (build, flatten, both traces) back to back; the same step as the timed region",
                     "clocks": clk2}

    # ---- the timed build's SAH against the oracle's, outside the timed region ----
    sah_check = None
    gold = golden_c2() if n_tris == N_TRIS else None
    if gold is not None:
        step()
        got_tree = float(plan.tree().sah())
        got_col = plan.sah()
        sah_check = {"tree_sah": got_tree, "oracle_tree_sah": gold["tree_sah"],
                     "collapsed_sah": float(got_col), "oracle_collapsed_sah": gold["collapsed_sah"],
                     "equal": bool(np.float32(got_tree) == np.float32(gold["tree_sah"])
                                   and np.float32(got_col) == np.float32(gold["collapsed_sah"]))}

    # ---- standalone refit of a resident LBVH + ATRBVH(9,2) tree (the serving
    # primitive): atr_refit from the scene's device vertices, K repetitions
    # after warm-up (the first refit builds the topology's refit plan) ----
    refit = measure_refit(ctx, stream, scene, n_tris, world, reps=max(20, args.steps // 4))

    # ---- e2e through the public API from pinned host memory ----
    # Each step: atr_scene_create from pinned host vertices with the host scene
    # box (as the reference's SceneWrapper takes it) -> atr_build_lbvh ->
    # atr_optimize_atrbvh -> atr_collapse with the SAH read back to the host.
    # Several steps are in flight (--e2e-inflight, default 4), each on its own
    # library context (stream) driven by its own host thread, so uploads overlap
    # other steps' kernels and the host link stays busy.
    pinned = torch.from_numpy(v.reshape(-1)).pin_memory().numpy().reshape(v.shape)
    bmin_h, bmax_h = ab.scene_bounds(pinned)  # input preparation, outside the timed region
    e2e = None
    if not args.no_e2e:
        inflight = max(1, args.e2e_inflight)
        ctxs = [ctx] + [ab.Context(local) for _ in range(inflight - 1)]
        sahs: list[list[float]] = [[] for _ in range(inflight)]

        def e2e_step(c: "ab.Context", k: int) -> None:
            sc = ab.SceneWrapper(c, pinned, bmin_h, bmax_h)
            tree = ab.LBVHBuilder(False).BuildTree(sc)
            ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
            col, sah = ab.BVHTreeCollapser().Collapse(tree)  # synchronises this context, reads the SAH back
            sahs[k].append(float(sah))
            col.close()
            tree.close()
            sc.close()

        def e2e_run(total: int) -> float:
            counts = [total // inflight + (1 if k < total % inflight else 0) for k in range(inflight)]
            errors: list[BaseException] = []

            def worker(k: int) -> None:
                try:
                    for _ in range(counts[k]):
                        e2e_step(ctxs[k], k)
                except BaseException as ex:  # reported after the join
                    errors.append(ex)

            barrier(world)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ths = [threading.Thread(target=worker, args=(k,)) for k in range(inflight)]
            for th in ths:
                th.start()
            for th in ths:
                th.join()
            dt = time.perf_counter() - t0
            if errors:
                raise errors[0]
            return dt

        e2e_run(max(inflight, args.warmup))
        for k in range(inflight):
            sahs[k].clear()
        e2e_dt = max_over_ranks(e2e_run(args.steps), world)
        got = {np.float32(x) for k in range(inflight) for x in sahs[k]}
        e2e = {"value": world * n_tris * args.steps / e2e_dt / 1e6, "unit": "Mtri/s",
               "h2d_bytes_per_step": int(v.nbytes) + 24, "d2h_bytes_per_step": 8,
               "steps": args.steps, "seconds": e2e_dt,
               "path": "atr_scene_create(pinned host vertices, host scene box) -> atr_build_lbvh -> "
                       f"atr_optimize_atrbvh -> atr_collapse (SAH read back); {inflight} steps in flight on "
                       f"{inflight} contexts (streams), one host thread each",
               "collapsed_sah_values": sorted(float(x) for x in got)}
        for c in ctxs[1:]:
            c.close()

    peaks = _read_peaks()
    roof = {}
    for k, bpt in BYTES_PER_TRI.items():
        if ph_ms.get(k):
            roof[k] = n_tris * bpt / (ph_ms[k] * 1e-3) / 1e9
    # The dominant phase by time is ATRBVH: its kernels (phase A climb, level
    # lists, one launch per treelet level, dataflow top) are issue- and
    # latency-bound, so its HBM fraction is small; traffic is the ncu DRAM
    # bytes of the same phase scaled to this triangle count.
    # The dominant phase with an algorithmic byte count (ATRBVH on this workload).
    times = {k: v2 for k, v2 in ph_ms.items() if k in BYTES_PER_TRI}
    dominant = max(times, key=times.get)
    achieved = roof.get(dominant, 0.0)
    rl = {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
          "frac": achieved / peaks["hbm_gbs"], "peak_src": peaks["src"],
          "traffic": (n_tris * ATRBVH_DRAM_BYTES_PER_TRI / 1e9 if dominant == "atrbvh" else None),
          "traffic_unit": "GB per step (ncu DRAM bytes, scaled)",
          "algorithmic_gb": n_tris * BYTES_PER_TRI.get(dominant, 0.0) / 1e9,
          "note": "issue/latency-bound phase (ncu: ~50-70% issue active, long-scoreboard stalls)"}
    out = {
        "metric": METRIC,
        "value": world * n_tris / (build_ms_max * 1e-3) / 1e6,
        "unit": "Mtri/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Philox: clustered scene + pinhole/diffuse rays)",
        "config": clustered_config(n_tris, world, rays_per_step),
        "mrays_per_s": world * rays_per_step / (trace_ms_max * 1e-3) / 1e6 if trace_ms_max else None,
        "phase_ms": {k: round(x, 4) for k, x in ph_ms.items()},
        "build_ms": build_ms_max,
        "phase_gbs": {k: round(x, 1) for k, x in roof.items()},
        "roofline": rl,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "graph_launches_per_step": 1,
        "timing": {"value": "Morton through collapse, the plan's two CUDA events recorded inside the replayed graph, "
                            "mean of K",
                   "phase_ms": "per-phase CUDA events inside the same plan's graph captured with phase marks, mean of "
                               "replays after the timed steps (the marks' event nodes are left out of the timed "
                               "graph); trace: events around both trace launches of the K timed steps"},
        "clocks": clk,
        "sustained": sustained,
        "sah_check": sah_check,
        "refit": refit,
    }
    plan.close()
    scene.close()
    del rays, res, bounce, res2
    torch.cuda.synchronize()
    if world == 1 and not args.no_batch:
        out["batch"] = measure_batch(ctx, stream, world, rank, device=local, steps=5, warmup=2, plain_reps=2,
                                     autotune=False, e2e=False)
    if world == 1 and not args.no_serve and rank == 0:
        out["serving"] = measure_serve(rates=[500.0, 1000.0, 2000.0, 5000.0], requests=1000, pool_size=16,
                                       lanes=args.lanes, device=local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


def measure_refit(ctx, stream, scene, n_tris: int, world: int, reps: int) -> dict:
    """Device time of atr_refit on a resident LBVH + ATRBVH(9,2) tree of the scene
    (CUDA events on the library's stream, mean of reps after three warm-up
    refits), as GB/s of the refit's algorithmic bytes."""
    import torch
    import atrbvh_b200 as ab
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    for _ in range(3):
        ab.Refit(tree, scene)
    ctx.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        ab.Refit(tree, scene)
    e1.record(stream)
    ctx.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / reps, world)
    tree.close()
    peaks = _read_peaks()
    gbs = n_tris * REFIT_BYTES_PER_TRI / (ms * 1e-3) / 1e9
    return {"ms": ms, "mtri_per_s": world * n_tris / (ms * 1e-3) / 1e6, "gbs": gbs,
            "frac_of_hbm": gbs / peaks["hbm_gbs"], "bytes_per_tri": REFIT_BYTES_PER_TRI, "reps": reps,
            "tree": "LBVH 30-bit + ATRBVH(9,2) of the workload scene, refit in place from its device vertices"}


BATCH_MESHES = 4096
BATCH_MIN, BATCH_MAX = 256, 262144
BATCH_WORKLOAD = ("4096 meshes, triangle counts log-uniform in [256, 262144] (seed 0), each a uniform-centroid "
                  "scene (vertex offsets N(0, 0.005^2)) rescaled into its own random unit box: LBVH 30-bit + "
                  "ATRBVH(9,2) per mesh, segmented batch build replayed from a CUDA graph vs per-mesh plain launches")


def _cuda_ms(stream, fn, reps: int) -> list[float]:
    """Device time of fn() per repetition (CUDA events on the library's stream)."""
    import torch
    out = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def measure_batch(ctx, stream, world, rank, *, device: int = 0, meshes: int = BATCH_MESHES, steps: int = 5,
                  warmup: int = 2, plain_reps: int = 3, autotune: bool = True, e2e: bool = True) -> dict:
    """Segmented batched builds of the 4096-mesh workload against per-mesh
    plain launches of the same library on the same GPU.  The trees are equal,
    so the SAH is equal: every 64th mesh's SAH is compared bit for bit."""
    import torch
    import atrbvh_b200 as ab
    from atrbvh_b200.shard import rank_meshes
    sizes_all = ab.gen_batch_sizes(meshes, BATCH_MIN, BATCH_MAX, 0)
    v_all = ab.gen_batch_scene(sizes_all, 0)
    total_tris = int(sizes_all.sum())
    if world > 1:
        # Meshes are independent: each rank builds its share (no collective on the data path).
        mine = rank_meshes(sizes_all, world, rank)
        off_all = np.concatenate([[0], np.cumsum(sizes_all, dtype=np.uint64)])
        v = np.ascontiguousarray(np.concatenate([v_all[off_all[m]:off_all[m + 1]] for m in mine]))
        sizes = np.ascontiguousarray(sizes_all[mine])
        del v_all
    else:
        v, sizes = v_all, sizes_all
    off = np.concatenate([[0], np.cumsum(sizes, dtype=np.uint64)]).astype(np.uint32)
    batch = ab.Batch(ctx, v, off)

    def build_batched():
        batch.build(1, 9, 2, graph=True)

    for _ in range(warmup):
        build_batched()
    ctx.synchronize()
    barrier(world)
    clocks = ClockSampler(device, interval_ms=50)
    clocks.start()
    l0 = ctx.launch_count()
    bt = _cuda_ms(stream, build_batched, steps)
    launches = (ctx.launch_count() - l0) // max(1, steps)
    clk = clocks.stop()
    sah_b = batch.sah()

    # Autotuned arm: per-class treelet/iterations at SAH no worse than
    # ATRBVH(9,2), ATRBVH block size and sort digit width of the dominant class.
    tuned = None
    if autotune:
        # Classes tuned on samples of up to 4M triangles, the table then checked
        # on this batch against the defaults and kept only if faster.
        w0, b0 = ctx.get_tuning(ab.TUNE_ATR_WARPS), ctx.get_tuning(ab.TUNE_SORT_BITS)
        t0 = time.perf_counter()
        table, outcome = ab.batch_autotune(ctx, batch, sample_triangles=1 << 22, reps=3)
        tune_s = time.perf_counter() - t0
        for _ in range(warmup):
            build_batched()
        tt = _cuda_ms(stream, build_batched, steps)
        sah_t = batch.sah()
        t_ms = max_over_ranks(statistics.median(tt), world)
        tuned = {"mtri_per_s": total_tris / (t_ms * 1e-3) / 1e6, "ms": t_ms,
                 "sah_ratio_vs_atrbvh_9_2": float(np.sum(sah_t, dtype=np.float64) / np.sum(sah_b, dtype=np.float64)),
                 "tuning_seconds": tune_s, "kept": bool(outcome["kept"]),
                 "tuner_batch_ms": {"default": outcome["default_ms"], "tuned": outcome["tuned_ms"]},
                 "table": {str(c): {k: e[k] for k in ("treelet", "iterations", "atr_warps", "sort_bits", "sah_ratio")}
                           for c, e in table.classes().items()}}
        batch.set_params(None)
        ctx.set_tuning(ab.TUNE_ATR_WARPS, w0)
        ctx.set_tuning(ab.TUNE_SORT_BITS, b0)

    # Per-mesh plain launches: one scene per mesh made up front (like the
    # batch's own upload), then LBVH + ATRBVH per mesh in the timed loop.
    scenes = [ab.SceneWrapper(ctx, np.ascontiguousarray(v[off[m]:off[m + 1]])) for m in range(len(sizes))]
    ctx.synchronize()

    def build_plain():
        for sc in scenes:
            t = ab.LBVHBuilder(False).BuildTree(sc)
            ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(t)
            t.close()

    build_plain()
    ctx.synchronize()
    pt = _cuda_ms(stream, build_plain, max(1, plain_reps))
    sah_equal = True
    checked = 0
    for m in range(0, len(sizes), 64):
        t = ab.LBVHBuilder(False).BuildTree(scenes[m])
        ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(t)
        sah_equal &= bool(np.float32(t.sah()) == np.float32(sah_b[m]))
        checked += 1
        t.close()
    for sc in scenes:
        sc.close()
    e2e_t = []
    if e2e:
        # pinned host vertices -> atr_batch_create -> build -> per-mesh SAH on the host.
        pinned = torch.from_numpy(v.reshape(-1)).pin_memory().numpy().reshape(v.shape)
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b2 = ab.Batch(ctx, pinned, off)
            b2.build(1, 9, 2)
            b2.sah()
            e2e_t.append(time.perf_counter() - t0)
            b2.close()
        del pinned
    batch.close()
    b_ms = max_over_ranks(statistics.median(bt), world)
    p_ms = max_over_ranks(statistics.median(pt), world)
    return {"workload": BATCH_WORKLOAD, "meshes": len(sizes_all), "triangles": total_tris,
            "batched_mtri_per_s": total_tris / (b_ms * 1e-3) / 1e6, "batched_ms": b_ms, "batched_steps": steps,
            "plain_mtri_per_s": total_tris / (p_ms * 1e-3) / 1e6, "plain_ms": p_ms, "plain_reps": max(1, plain_reps),
            "batched_vs_plain": p_ms / b_ms, "sah_equal_checked_meshes": checked, "sah_equal": sah_equal,
            "autotuned": tuned, "gpu_launches_per_batched_step": int(launches), "clocks": clk,
            "e2e_s": (max_over_ranks(statistics.median(e2e_t), world) if e2e_t else None),
            "h2d_bytes": int(v.nbytes), "timing": "CUDA events on the library stream, median of the timed steps"}


def run_batch(args, world, rank, local):
    import torch
    import atrbvh_b200 as ab
    torch.cuda.set_device(local)
    ctx = ab.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    r = measure_batch(ctx, stream, world, rank, device=local, meshes=args.meshes, steps=args.steps,
                      warmup=args.warmup,
                      plain_reps=min(args.steps, 3), autotune=not args.no_autotune, e2e=not args.no_e2e)
    total = r["triangles"]
    out = {
        "metric": METRIC, "value": r["batched_mtri_per_s"], "unit": "Mtri/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["batched_ms"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox)",
        "config": {"workload": BATCH_WORKLOAD, "meshes": r["meshes"], "triangles": total, "treelet": 9,
                   "iterations": 2, "morton_bits": 30,
                   "parallelism": "meshes sharded by size over ranks" if world > 1 else "one GPU",
                   "l2": f"inputs larger than L2 ({total * 48 / 1e9:.1f} GB of vertices)"},
        "plain_mtri_per_s": r["plain_mtri_per_s"], "plain_ms": r["plain_ms"],
        "batched_vs_plain": r["batched_vs_plain"],
        "sah_equal_checked_meshes": r["sah_equal_checked_meshes"], "sah_equal": r["sah_equal"],
        "autotuned": r["autotuned"], "gpu_launches": r["gpu_launches_per_batched_step"] * args.steps,
        "e2e": {"value": (total / r["e2e_s"] / 1e6) if r["e2e_s"] else None, "unit": "Mtri/s",
                "h2d_bytes_per_step": r["h2d_bytes"], "d2h_bytes_per_step": 4 * r["meshes"],
                "path": "atr_batch_create(pinned host vertices) -> atr_batch_build -> atr_batch_sah"},
        "clocks": r["clocks"],
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()


SERVE_WORKLOAD = ("serving loop: Poisson arrivals; each request builds a mesh (log-uniform 1k-2M triangles, "
                  "uniform-centroid scene) or refits a resident one after N(0, 0.001^2) vertex jitter, then traces "
                  "64k-1M random rays; 120 GB device-memory budget")


def measure_serve(*, rates, requests: int, pool_size: int, lanes: int, device: int = 0,
                  pinned: bool = True, warmup_requests: int = 64) -> list[dict]:
    """The serving loop under Poisson arrivals: p50/p99 request latency beside
    build and trace throughput, one record per arrival rate.  With pinned, the
    requests' vertex, ray and result buffers are page-locked host memory,
    which the server copies to and from the device directly."""
    import atrbvh_b200 as ab
    rng = np.random.default_rng(0)
    host = ab.pinned_like if pinned else (lambda a: a)
    pool = []
    for k in range(pool_size):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(2_000_000))))
        v = ab.gen_scene(ab.SCENE_UNIFORM, n, 1000 + k)
        j = (v + rng.normal(0.0, 0.001, v.shape).astype(np.float32)).astype(np.float32)
        j[:, :, 3] = 0.0
        p = v[:, :, :3].reshape(-1, 3)
        nr = int(np.exp(rng.uniform(np.log(65536), np.log(1 << 20))))
        rays = ab.gen_rays_random(nr, p.min(0), p.max(0), seed=2000 + k)
        pool.append((host(v), host(j), host(rays)))
    max_rays = max(len(r) for _, _, r in pool)
    n_outs = 2 * lanes * 32 + 8
    outs = [host(np.zeros((max_rays, 4), np.int32)) for _ in range(n_outs)]
    rows = []
    for rate in rates:
        srv = ab.Server(device=device, hbm_budget=120 << 30, lanes=lanes, max_batch_requests=32,
                        max_batch_triangles=1 << 25)
        # Warm-up: every lane's context, pool and staging reach steady state
        # before the arrival clock starts (these requests are not timed).
        warm = []
        for i in range(warmup_requests):
            k = i % len(pool)
            v, _, rays = pool[k]
            warm.append(srv.submit(ab.REQ_BUILD, 10 ** 9 + i, v, rays, outs[i % len(outs)], keep_resident=False))
        for t in warm:
            srv.wait(t)
        st0 = srv.stats()
        arrivals = np.cumsum(rng.exponential(1.0 / rate, requests))
        resident: list[int] = []
        tickets = []
        latencies: list[float] = []
        t0 = time.perf_counter()
        for i in range(requests):
            delay = arrivals[i] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            k = int(rng.integers(len(pool)))
            v, j, rays = pool[k]
            out = outs[i % len(outs)]
            keep = False
            if resident and rng.random() < 0.3:
                mid = resident[int(rng.integers(len(resident)))]
                kind, verts = ab.REQ_REFIT, pool[mid % len(pool)][1]
                rays = pool[mid % len(pool)][2]
            else:
                mid = i * len(pool) + k  # mesh id encodes its pool entry
                kind, verts = ab.REQ_BUILD, v
                if len(resident) < 64:  # the first 64 builds stay resident for refits
                    resident.append(mid)
                    keep = True
            tickets.append(srv.submit(kind, mid, verts, rays, out, keep_resident=keep))
            # Keep the output buffers' reuse distance: wait for old requests.
            if len(tickets) >= len(outs) - 4:
                latencies.append(srv.wait(tickets.pop(0))["latency_ms"])
        while tickets:
            latencies.append(srv.wait(tickets.pop(0))["latency_ms"])
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        lat = np.sort(np.asarray(latencies))
        pct = lambda q: float(lat[min(len(lat) - 1, int(np.ceil(q * len(lat))) - 1)])  # noqa: E731
        rows.append({"rate_per_s": rate, "requests": requests, "p50_ms": pct(0.50), "p99_ms": pct(0.99),
                     "mean_ms": float(lat.mean()), "max_ms": float(lat[-1]),
                     "completed": st["completed"] - st0["completed"], "failed": st["failed"] - st0["failed"],
                     "builds": st["builds"] - st0["builds"], "refits": st["refits"] - st0["refits"],
                     "build_mtri_per_s": (st["triangles_built"] - st0["triangles_built"]) / wall / 1e6,
                     "trace_mrays_per_s": (st["rays_traced"] - st0["rays_traced"]) / wall / 1e6, "wall_s": wall,
                     "served_per_s": requests / wall, "warmup_requests": warmup_requests,
                     "lane_batches": st["lane_batches"], "max_batch_requests_seen": st["max_batch_requests_seen"],
                     "overlap_fraction": st["overlap_fraction"], "peak_gb": st["peak_bytes"] / 1e9,
                     "host_copy_ms": st["host_copy_ms"] - st0["host_copy_ms"],
                     "lane_batch_ms": st["lane_batch_ms"] - st0["lane_batch_ms"],
                     "pinned_request_buffers": pinned})
    return rows


def run_serve(args, world, rank, local):
    rows = measure_serve(rates=[float(x) for x in args.rates.split(",")], requests=args.requests,
                         pool_size=args.pool, lanes=args.lanes, device=local)
    for r in rows:
        out = {
            "metric": METRIC, "value": r["p99_ms"], "unit": "ms (p99 request latency)", "n_gpus": 1,
            "steps": args.requests, "warmup": 0, "ms_per_step": r["wall_s"] * 1e3 / args.requests,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": SERVE_WORKLOAD, "requests": args.requests, "rate_per_s": r["rate_per_s"],
                       "pool_meshes": args.pool, "lanes": args.lanes},
            **{k: v for k, v in r.items() if k not in ("rate_per_s", "requests")},
        }
        print(json.dumps(out), flush=True)


SWEEP_WORKLOAD = ("16,777,216 uniform-centroid triangles (vertex offsets N(0, 0.005^2)), seed 0: LBVH, "
                  "TRBVH(7,3), ATRBVH(5/7/9 x 1-3); 8,388,608 random rays (origins in the scene box, "
                  "directions uniform on the sphere)")


def run_sweep(args, world, rank, local):
    """Quality/speed sweep: SAH, per-phase Mtri/s and Mrays/s per optimiser."""
    import torch
    import atrbvh_b200 as ab
    torch.cuda.set_device(local)
    ctx = ab.Context(local)
    n = args.sweep_triangles
    v = ab.gen_scene(ab.SCENE_UNIFORM, n, 0)
    scene = ab.SceneWrapper(ctx, v)
    mn, mx = scene.bounds()
    rays_h = ab.gen_rays_random(1 << 23, mn, mx, seed=0)
    nr = len(rays_h)
    with torch.cuda.stream(torch.cuda.ExternalStream(ctx.stream)):
        rays = torch.from_numpy(rays_h.reshape(-1)).cuda()
        res = torch.empty(nr * 4, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    variants = [("lbvh", 0, 0, 0)] + [("trbvh", 2, 7, 3)] + [("atrbvh", 1, t, i) for t in (5, 7, 9) for i in (1, 2, 3)]
    rows = []
    for name, opt, ts, it in variants:
        ph_all = []
        for rep in range(args.warmup + args.steps):
            ctx.set_timing(True)
            tree = ab.LBVHBuilder(False).BuildTree(scene)
            if opt == 1:
                ab.AgglomerativeTreeletOptimizer(ts, it).Optimize(tree)
            elif opt == 2:
                ab.TRBVHOptimizer(ts, it).Optimize(tree)
            col, csah = ab.BVHTreeCollapser().Collapse(tree)
            bvh = ab.CudaBVH(col, scene)
            bvh.trace(rays.data_ptr(), nr, res.data_ptr())
            ctx.synchronize()
            ph = ctx.phase_times()
            ctx.set_timing(False)
            sah = tree.sah()
            bvh.close(); col.close(); tree.close()
            if rep >= args.warmup:
                d = {}
                for k2, ms in ph:
                    d[k2] = d.get(k2, 0.0) + ms
                ph_all.append(d)
        med = {k2: statistics.median(x[k2] for x in ph_all) for k2 in ph_all[0]}
        build_ms = sum(med.get(k2, 0.0) for k2 in ("morton", "sort", "build", "atrbvh", "trbvh"))
        rows.append({"optimizer": name, "treelet": ts, "iterations": it, "sah": sah, "collapsed_sah": csah,
                     "build_ms": build_ms, "build_mtri_per_s": n / (build_ms * 1e-3) / 1e6,
                     "phase_ms": {k2: round(x, 4) for k2, x in med.items()},
                     "phase_mtri_per_s": {k2: round(n / (x * 1e-3) / 1e6, 1) for k2, x in med.items() if k2 != "trace"},
                     "mrays_per_s": nr / (med["trace"] * 1e-3) / 1e6})
    best = max(rows, key=lambda r: r["build_mtri_per_s"] if r["optimizer"] == "atrbvh" and r["treelet"] == 9
               and r["iterations"] == 2 else -1)
    out = {"metric": METRIC, "value": best["build_mtri_per_s"], "unit": "Mtri/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": best["build_ms"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox)",
           "config": {"workload": SWEEP_WORKLOAD, "triangles": n, "rays": nr, "value_of": "ATRBVH(9,2) build"},
           "sweep": rows}
    print(json.dumps(out), flush=True)


REFIT_WORKLOAD = ("clustered scene (as the default workload): LBVH 30-bit + ATRBVH(9,2) once, then atr_refit of "
                  "the resident tree from its device vertices per step (the refit plan is built by the second refit, "
                  "inside the warm-up)")


def run_refit(args, world, rank, local):
    """Standalone refit of a resident tree: one atr_refit per step."""
    import torch
    import atrbvh_b200 as ab
    torch.cuda.set_device(local)
    ctx = ab.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    n = args.triangles
    scene = ab.SceneWrapper(ctx, ab.gen_scene(ab.SCENE_CLUSTERED, n, 0))
    tree = ab.LBVHBuilder().BuildTree(scene)
    ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
    for _ in range(max(args.warmup, 3)):
        ab.Refit(tree, scene)
    ctx.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ab.Refit(tree, scene)
    e1.record(stream)
    ctx.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    peaks = _read_peaks()
    gbs = n * REFIT_BYTES_PER_TRI / (ms * 1e-3) / 1e9
    if rank == 0:
        print(json.dumps({"metric": "refit Mtri/s", "value": world * n / (ms * 1e-3) / 1e6, "unit": "Mtri/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic (seeded Philox)",
                          "config": {"workload": REFIT_WORKLOAD, "triangles": n},
                          "roofline": {"kernel": "k_refit_level", "bound": "hbm", "achieved": gbs,
                                       "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": gbs / peaks["hbm_gbs"],
                                       "peak_src": peaks["src"], "bytes_per_tri": REFIT_BYTES_PER_TRI}}), flush=True)
    tree.close()
    scene.close()
    ctx.close()


SPLIT_WORKLOAD = ("sliver scene: the uniform-centroid scene with 10% of its triangles replaced by slivers (length "
                  "0.2-0.6 along random directions, width 0.002; seeded): triangle splitting at ratios 0-1, "
                  "primitive-box LBVH 30-bit + ATRBVH(9,2) + collapse, SAH and build times against the plain build")


def sliver_scene(n: int, seed: int = 9):
    import atrbvh_b200 as ab
    v = ab.gen_scene(ab.SCENE_UNIFORM, n, seed).copy()
    rng = np.random.default_rng(seed)
    k = n // 10
    idx = rng.choice(n, size=k, replace=False)
    p0 = rng.uniform(0.0, 1.0, (k, 3)).astype(np.float32)
    d = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = np.cross(d, rng.normal(size=(k, 3)))
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    length = rng.uniform(0.2, 0.6, (k, 1))
    v[idx, 0, :3] = p0
    v[idx, 1, :3] = (p0 + length * d).astype(np.float32)
    v[idx, 2, :3] = (p0 + 0.002 * w).astype(np.float32)
    v[:, :, 3] = 0
    return np.ascontiguousarray(v)


def run_split(args, world, rank, local):
    """Triangle splitting on a scene of slivers: SAH and device times of split
    + primitive-box LBVH + ATRBVH(9,2) + collapse against the plain build."""
    import torch
    import atrbvh_b200 as ab
    torch.cuda.set_device(local)
    ctx = ab.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    n = args.triangles
    v = sliver_scene(n)
    mn, mx = ab.scene_bounds(v)
    scene = ab.SceneWrapper(ctx, v, mn, mx)
    rows = []
    for ratio in (None, 0.1, 0.3, 1.0):
        times = []
        for rep in range(args.warmup + args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if ratio is None:
                tree = ab.LBVHBuilder().BuildTree(scene)
                prims = n
            else:
                bmin, bmax, data = ab.split_triangles(scene, ratio)  # synchronises to read the count
                tree = ab.build_lbvh_split(ctx, bmin, bmax, data, mn, mx)
                prims = int(data.shape[0])
            ab.AgglomerativeTreeletOptimizer(9, 2).Optimize(tree)
            col, csah = ab.BVHTreeCollapser().Collapse(tree)
            e1.record(stream)
            ctx.synchronize()
            if rep >= args.warmup:
                times.append(e0.elapsed_time(e1))
            sah = tree.sah()
            col.close()
            tree.close()
        ms = statistics.median(times)
        rows.append({"split_ratio": ratio, "primitives": prims, "sah": sah, "collapsed_sah": csah, "ms": ms,
                     "mtri_per_s": n / (ms * 1e-3) / 1e6})
    plain = rows[0]
    for r in rows:
        r["sah_vs_plain"] = r["sah"] / plain["sah"]
    best = min(rows[1:], key=lambda r: r["sah"])
    if rank == 0:
        print(json.dumps({"metric": "ATRBVH SAH with triangle splitting (lower is better)", "value": best["sah"],
                          "unit": "SAH", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": best["ms"], "higher_is_better": False, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                          "config": {"workload": SPLIT_WORKLOAD, "triangles": n}, "rows": rows}), flush=True)
    scene.close()
    ctx.close()


def run_reference(args, world, rank, local):
    """The host-core pipeline on the whole workload scene, one build per step.
    The reference has no CPU implementation of this path, and its CUDA build
    is not run here; the checker's restatement of the same pipeline
    (LBVH 30-bit + ATRBVH(9,2) + collapse) stands in for it.  Nothing from the
    product library is loaded: the scene comes from the checker's own
    generator (the same bits as the product's)."""
    if rank != 0:
        return
    import oracle as O
    v = O.gen_scene(O.SCENE_CLUSTERED, N_TRIS, 0)
    threads = O.max_threads()
    for _ in range(args.warmup):
        cpu_pipeline(v, threads)
    secs = [cpu_pipeline(v, threads) for _ in range(args.steps)]
    mean_s = statistics.mean(secs)
    value = N_TRIS / mean_s / 1e6
    out = {
        "metric": METRIC, "value": value, "unit": "Mtri/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Philox: clustered scene + pinhole/diffuse rays)",
        "impl": "reference",
        "config": clustered_config(N_TRIS, world, WIDTH * HEIGHT * 2),
        "best_of_steps": N_TRIS / min(secs) / 1e6,
        "cpu_baseline": {"value": value, "unit": "Mtri/s", "cores": threads, "kind": "port",
                         "sample": f"the whole {N_TRIS}-triangle workload scene per step (no sample): "
                                   f"LBVH+ATRBVH(9,2)+collapse on {threads} host threads, mean of {args.steps} steps "
                                   f"after {args.warmup} warm-ups"},
        "e2e": {"value": value, "unit": "Mtri/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": {
            "unavailable": "the reference's ATRBVH CUDA kernel, compiled here for sm_100a, did not terminate on a "
                           "4,096-triangle input on this pool (unfenced cross-SM reads of treelet rewrites); it is "
                           "not run again"},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-inflight", type=int, default=4, help="e2e: steps in flight (one context and thread each)")
    ap.add_argument("--no-batch", action="store_true", help="default line: skip the 4096-mesh batched-vs-plain keys")
    ap.add_argument("--no-serve", action="store_true", help="default line: skip the serving p50/p99 keys")
    ap.add_argument("--sustain-s", type=float, default=1.0,
                    help="default line: seconds of back-to-back steps timed after the K steps, with their own clocks")
    ap.add_argument("--triangles", type=int, default=N_TRIS,
                    help="scene size (default: the workload's 4,194,304); smaller values are for profiling")
    ap.add_argument("--workload", default="clustered", choices=["clustered", "batch", "serve", "sweep", "refit",
                                                                "split"],
                    help="clustered: 4.2M-triangle build+trace (the default line); batch: 4096-mesh segmented "
                         "build vs per-mesh launches; serve: the request loop; sweep: 16.8M-triangle optimiser sweep")
    ap.add_argument("--meshes", type=int, default=BATCH_MESHES, help="batch: number of meshes")
    ap.add_argument("--no-autotune", action="store_true", help="batch: skip the autotuned arm")
    ap.add_argument("--requests", type=int, default=20000, help="serve: requests per arrival rate")
    ap.add_argument("--rates", default="100,200,500,1000,2000,5000",
                    help="serve: comma-separated arrival rates per second")
    ap.add_argument("--lanes", type=int, default=3, help="serve: concurrent lanes")
    ap.add_argument("--pool", type=int, default=48, help="serve: distinct meshes drawn by the requests")
    ap.add_argument("--sweep-triangles", type=int, default=1 << 24, help="sweep: scene size")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, local)
        elif args.workload == "batch":
            run_batch(args, world, rank, local)
        elif args.workload == "serve":
            if rank == 0:
                run_serve(args, world, rank, local)
        elif args.workload == "sweep":
            if rank == 0:
                run_sweep(args, world, rank, local)
        elif args.workload == "refit":
            run_refit(args, world, rank, local)
        elif args.workload == "split":
            if rank == 0:
                run_split(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
