#!/usr/bin/env python
"""Benchmark of the B200 n-space path tracer: paths/s on the n = 4 measured scene.

Workload (the configuration the metric is quoted on): the boundary of the convex hull of 100,000
seeded points on the unit 3-sphere (675,456 tetrahedra) above a 4-parallelotope floor
[-4,4]^3 x [-1.1,-1], a point light at (2,2,2,3), parallel projection onto a 128^3 screen, 16 samples
per pixel (27 after stratification), recursion depth 5, FP32 with the FP64 re-test.  One step = one
full frame (56,623,104 camera paths).  The scene arrays (~400 MB) exceed the 126 MB L2, so no L2 flush
is needed between steps.

--impl ours (default): the sm_100a wavefront through the C ABI.  value: paths/s, device-timed with
CUDA events on the scene's stream over K steps (max over ranks); e2e: the same through the public API
with the scene's arrays copied from pinned host memory and the image read back every step.
--impl reference: the reference painter (oracle/_ref, compiled from the reference's own sources) on
the host's cores, each step a seeded random pixel sample of the same frame.

On one GPU the line also carries (skip with --no-extras):
  per_n: the n = 3 (400^2, 16 spp, 20,480 triangles) and n = 5 (48^4, 16 spp after stratification,
      1,541,774 4-simplices) configurations, measured the same way over 5 frames;
  denoise_time_to_rmse_1e-2: per configuration, the time a whole frame needs to reach relative RMSE
      1e-2 (on the centred window, against a 64k-sample render of it) plain and with the learned
      denoiser (committed weights), on the k^(n-1) sample grid; the plain time fitted to the target.

Multi-GPU (torchrun): every rank renders the whole frame with its own sample range (weak scaling);
the per-pixel sums are combined with one NCCL all-reduce after the timed region.
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

CONFIGS = {"n3": "n3", "n4": "n4", "n5": "n5", "batch": "batch"}
def metric_name(n: int) -> str:
    return f"paths/s per n (n={n} plain tracer)"


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_work(n: int, facet_tests: int, box_steps: int, descent: int) -> tuple[int, int]:
    """Bytes and flops of the reference algorithm's tree walk for the given counts (per unit:
    a descent level reads one box, 2n floats; a visited leaf one exit slab, 2n floats; a facet test
    one index and one simplex record, n^2 + 2n - 1 floats; flops: 2n per level, 6n per slab,
    2n^2 + 4n per facet test)."""
    b = descent * 2 * n * 4 + box_steps * 2 * n * 4 + facet_tests * ((n * n + 2 * n - 1) * 4 + 4)
    f = descent * 2 * n + box_steps * 6 * n + facet_tests * (2 * n * n + 4 * n)
    return b, f


def pixel_sample(screen, count: int, rng) -> np.ndarray:
    """`count` distinct random pixels of the screen as (count, n-1) coordinates."""
    npix = int(np.prod(screen))
    lin = np.sort(rng.choice(npix, count, replace=False))
    return np.stack([(lin // int(np.prod(screen[:j]))) % screen[j] for j in range(len(screen))], axis=1)


def cpu_baseline(spec: dict, paths_target: int, threads: int) -> dict:
    """The reference painter (its own -Ofast build) on the host cores over a seeded random pixel
    sample of the frame."""
    from math_b200 import scenes
    from oracle import checkers

    n = spec["n"]
    screen = spec["projector"]["screen"]
    npix = int(np.prod(screen))
    spp_eff = scenes.effective_spp(n, spec["spp"])
    count = int(min(npix, max(1000, paths_target // spp_eff)))
    px = pixel_sample(screen, count, np.random.default_rng(12345))
    if checkers.Reference.available(fast=True):
        ref = checkers.Reference(fast=True)
        _, st = ref.paint(spec, dbl=False, seed=1, threads=threads, pixels=px, store=False)
        return {"value": st["sample_count"] / st["seconds"], "unit": "paths/s", "cores": threads,
                "kind": "reference", "seconds": st["seconds"], "build": ref.flags,
                "sample": f"{count} random pixels of the {'x'.join(map(str, screen))} frame x {spp_eff} spp "
                          f"= {st['sample_count']} paths, paint<{n},float>() ({ref.flags}) with {threads} threads"}
    port = checkers.Port()
    _, st = port.paint(spec, dbl=False, threads=threads, pixels=px)
    return {"value": st["paths"] / st["seconds"], "unit": "paths/s", "cores": threads, "kind": "port",
            "seconds": st["seconds"],
            "sample": f"{count} random pixels x {spp_eff} spp with the C restatement, {threads} threads"}


def run_reference(args) -> None:
    """The reference painter alone in this process: the scene's mesh comes from scipy's Qhull (the
    same facet set as the library's hull) and the sample sizes from a Python restatement, so that
    nothing of math_b200's native code is loaded; the painter is the reference's own -Ofast build."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from math_b200 import scenes
    from oracle import checkers

    if not checkers.Reference.available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/fast/libref_painter.so is not built"}))
        return
    spec = scenes.config(args.config, hull="qhull")
    threads = os.cpu_count() or 1
    n = spec["n"]
    ref = checkers.Reference(fast=True)
    screen = spec["projector"]["screen"]
    npix = int(np.prod(screen))
    spp_eff = scenes.effective_spp(n, spec["spp"])
    count = min(npix, args.cpu_paths // spp_eff)
    rng = np.random.default_rng(7)
    total_paths, total_s = 0, 0.0
    for step in range(args.warmup + args.steps):
        px = pixel_sample(screen, count, rng)
        _, st = ref.paint(spec, dbl=False, seed=step + 1, threads=threads, pixels=px, store=False)
        if step >= args.warmup:
            total_paths += st["sample_count"]
            total_s += st["seconds"]
    value = total_paths / total_s
    sample = (f"per step {count} random pixels of the {'x'.join(map(str, screen))} frame x {spp_eff} spp, "
              f"paint<{n},float>() of the reference ({ref.flags}) with {threads} threads; mesh: the same "
              f"facet set from scipy's Qhull")
    print(json.dumps({
        "impl": "reference", "metric": metric_name(spec["n"]), "value": value, "unit": "paths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(spec, args),
        "mesh": mesh_block(spec, "scipy Qhull of the same points (the library's exact hull differs in the "
                                 "triangulation of a few near-degenerate regions)"),
        "cpu_baseline": {"value": value, "unit": "paths/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


WORKLOAD_MESH = {
    "n3": "icosphere subdivided 5 times (20,480 triangles)",
    "n4": "hull boundary of 100,000 seeded points on S^3 (tetrahedra)",
    "n5": "hull boundary of 50,000 seeded points on S^4 without a cap of angular radius 0.5 (4-simplices)",
}


def config_block(spec: dict, args) -> dict:
    """The workload, identical in both arms (what differs between them goes in mesh_block)."""
    n = spec["n"]
    return {"workload": f"n={n} plain tracer: {WORKLOAD_MESH[args.config]} + floor + point light, "
                        f"parallel projection {'x'.join(map(str, spec['projector']['screen']))}, "
                        f"{spec['spp']} spp, depth {spec['max_depth']}, FP32 + FP64 re-test",
            "n": n, "screen": spec["projector"]["screen"], "spp": spec["spp"],
            "max_depth": spec["max_depth"], "seed": spec["seed"],
            "l2": "scene arrays larger than the 126 MB L2; no flush between steps"}


def mesh_block(spec: dict, hull: str) -> dict:
    return {"facets": int(len(spec["facets"])), "vertices": int(len(spec["verts"])), "hull": hull}


def measure_plain(scene, spec: dict, args, steps: int, rank: int, world: int, local: int, dist,
                  e2e: bool = True) -> dict:
    """paths/s of the plain tracer on one built scene: autotuned pool, W warm-up frames (the last one
    with per-kernel device events), K timed frames between two events on the scene's stream (max over
    ranks), then K frames end to end through the public API."""
    import torch

    from math_b200 import distributed, scenes

    n = spec["n"]
    spp, depth = spec["spp"], spec["max_depth"]
    stream = torch.cuda.ExternalStream(scene.stream)
    # the library's autotuner picks the path-pool size and the iterations per graph launch from probe
    # passes of this frame (untimed; it clears the accumulator)
    tuned, _ = scene.autotune(spp, max_depth=depth, seed=spec["seed"])
    # every rank traces the same Philox stream; ranks take disjoint sample ranges (pass k of rank r
    # covers samples [(k * world + r) * spp_eff, + spp_eff)), so N ranks render N different passes
    spp_eff = scenes.effective_spp(n, spp)

    def offset(k: int) -> int:
        return distributed.sample_offset(rank, k, spp_eff, world)

    ropts = dict(max_depth=depth, seed=spec["seed"], pool_paths=tuned["pool_paths"],
                 graph_iterations=tuned["graph_iterations"], walk_chunk=tuned["walk_chunk"],
                 walk_small_leaf=tuned["walk_small_leaf"])

    # warm-up (the last one is also the per-kernel timing pass: device events around every launch)
    for _ in range(args.warmup - 1):
        scene.render(spp, **ropts)
    timed = scene.render(spp, **ropts, timing=True)
    scene.clear()

    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stats = []
    with ClockSampler(local) as clocks:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for k in range(steps):
            stats.append(scene.render(spp, **ropts, sample_offset=offset(k)))
        ev1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = ev0.elapsed_time(ev1)
    paths = sum(s["paths"] for s in stats)
    ms_all = torch.tensor([ms], dtype=torch.float64, device="cuda")
    paths_all = torch.tensor([paths], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(ms_all, op=dist.ReduceOp.MAX)
        dist.all_reduce(paths_all, op=dist.ReduceOp.SUM)
    ms_max = float(ms_all.item())
    out = {"value": float(paths_all.item()) / (ms_max / 1000.0), "ms_per_step": ms_max / steps, "steps": steps,
           "paths_per_step": paths // max(1, steps), "launches": sum(s["launches"] for s in stats),
           "device_errors": sum(s["error_bits"] for s in stats), "timed": timed, "tuned": tuned,
           "clocks": clocks.summary()}

    # combine the ranks' samples (disjoint sample ranges of one Philox stream) into one image: one NCCL
    # all-reduce of the per-pixel sums, after the timed region
    if dist:
        img, spp_done = scene.image()
        t0 = time.perf_counter()
        distributed.combine(img, spp_done)
        torch.cuda.synchronize()
        out["combine_ms"] = 1000 * (time.perf_counter() - t0)

    if e2e:
        # end to end through the public API: every step's scene arrays cross from pinned host memory
        # (double-buffered: step k+1's copy into the staging buffers runs on the scene's copy stream
        # while step k renders, then moves into the live arrays on the device), every step's image is
        # read back; wall clock around the calls, the first step's copy included
        scene.clear()
        host_img = torch.empty((scene.pixel_count, 3), dtype=torch.float32, pin_memory=True).numpy()
        # one untimed round of the upload path first: its first call creates the copy stream and
        # allocates the device staging buffers (set-up, not per-frame work)
        scene.upload_begin()
        scene.upload_commit()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_paths = 0
        h2d = scene.upload_begin()
        for k in range(steps):
            scene.upload_commit()
            if k + 1 < steps:
                scene.upload_begin()
            st = scene.render(spp, **ropts, sample_offset=offset(k))
            scene.image(out=host_img)
            e2e_paths += st["paths"]
        e2e_s = time.perf_counter() - t0
        e2e_all = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(e2e_all, op=dist.ReduceOp.MAX)
        out["e2e"] = {"value": e2e_paths * world / float(e2e_all.item()), "unit": "paths/s", "h2d_bytes_per_step": h2d,
                      "d2h_bytes_per_step": host_img.nbytes, "steps": steps}
    return out


def roofline(n: int, timed: dict, name: str, pool_paths: int, probes: dict | None = None) -> dict:
    """Roofline of the dominant walk kernel (the one with the larger device time) from the timing pass:
    algorithmic bytes per launch (the reference algorithm's work counters, algorithmic_work) over the
    launch's CUDA-event time, against the measured HBM copy peak."""
    peaks = measured_peaks()
    walks = {}
    for kind, prefix in (("extend", ""), ("shadow", "shadow_")):
        b, f = algorithmic_work(n, timed[prefix + "facet_tests"], timed[prefix + "box_steps"],
                                timed[prefix + "descent_levels"])
        launches_k = max(1, timed[kind + "_launches"])
        ms = timed[kind + "_ms"] / launches_k
        walks[kind] = {"bytes": b / launches_k, "flops": f / launches_k, "launch_ms": ms,
                       "achieved": (b / launches_k) / (ms / 1000.0) / 1e9 if ms > 0 else 0.0}
    dom = max(walks, key=lambda k: timed[k + "_ms"])
    # DRAM bytes per launch from an ncu capture (profiles/traffic.json), scaled by the algorithmic bytes
    # of this run's launches over those of the captured ones when the pool size differs (a launch's
    # traffic grows with the rays it processes)
    traffic = l2_traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            t = json.loads(tf.read_text())
            alg = t.get(f"{name}_{dom}_algorithmic_bytes_per_launch")
            scale = walks[dom]["bytes"] / alg if alg else None
            traffic = t.get(f"{name}_{dom}_bytes_per_launch")
            l2_traffic = t.get(f"{name}_{dom}_l2_bytes_per_launch")
            if scale is not None:
                traffic = traffic * scale if traffic is not None else None
                l2_traffic = l2_traffic * scale if l2_traffic is not None else None
        except Exception:
            traffic = l2_traffic = None
    achieved = walks[dom]["achieved"]
    launch_s = walks[dom]["launch_ms"] / 1000.0
    out = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
           "kernel": "k_shadow_refill" if dom == "shadow" else "k_extend_refill",
           "peak_source": peaks["source"], "algorithmic_bytes_per_launch": walks[dom]["bytes"],
           "algorithmic_flops_per_launch": walks[dom]["flops"], "launch_ms": walks[dom]["launch_ms"],
           "walk_algorithmic_gbs": {k: w["achieved"] for k, w in walks.items()}}
    if probes:
        # the other two ceilings of the walk: its L2 traffic (the ncu capture's L2 sectors per launch,
        # scaled like the DRAM traffic) against the L2 read rate, and its algorithmic FP32 flops against
        # the FMA rate, both peaks measured by the library's probe kernels (nt_probe_peaks)
        if l2_traffic is not None and launch_s > 0:
            a = l2_traffic / launch_s / 1e9
            out["l2"] = {"achieved": a, "peak": probes["l2_read_gbs"], "unit": "GB/s",
                         "frac": a / probes["l2_read_gbs"], "traffic": l2_traffic, "peak_source": "nt_probe_peaks"}
        if launch_s > 0:
            a = walks[dom]["flops"] / launch_s / 1e12
            out["fp32"] = {"achieved": a, "peak": probes["fp32_fma_tflops"], "unit": "TFLOP/s",
                           "frac": a / probes["fp32_fma_tflops"], "peak_source": "nt_probe_peaks"}
    return out


def measure_denoise(scene, n: int) -> dict:
    """The other half of the metric: time to relative RMSE <= 1e-2 against a 64k-sample render, plain
    versus denoised (the committed weights), on a held-out variation of the scene at its configuration
    screen (math_b200.train_denoiser.time_to_rmse)."""
    from math_b200 import denoise, train_denoiser

    den = denoise.Denoiser.load(ROOT / "math_b200" / "weights" / f"denoiser_n{n}.npz")
    r = train_denoiser.time_to_rmse(scene, den, n, 1e-2, seed=77 + n)

    def met(points):
        ok = [p for p in points if p["rmse"] <= 1e-2]
        return {"spp": ok[0]["spp"], "ms": 1000 * ok[0]["seconds"], "rmse": ok[0]["rmse"]} if ok else None

    return {"screen": r["screen"], "reference_window": r["reference_window"], "reference_spp": r["reference_spp"],
            "plain": met(r["plain"]), "denoised": met(r["denoised"]),
            "plain_fitted_ms": 1000 * r["plain_time_to_target_fitted"],
            "speedup": r["speedup"], "speedup_vs_fitted": r["speedup_vs_fitted"],
            "plain_points": [{"spp": p["spp"], "ms": 1000 * p["seconds"], "rmse": p["rmse"]} for p in r["plain"]],
            "denoised_points": [{"spp": p["spp"], "ms": 1000 * p["seconds"], "rmse": p["rmse"],
                                 "input_rmse": p["input_rmse"]} for p in r["denoised"]]}


def run_batch(args) -> None:
    """--config batch: the batched mixed workload (math_b200.batched): 64 seeded scenes of n = 3..6 in
    one CUDA graph per pass (nt_render_batch), tuned per dimension by nt_autotune; wall clock around
    each synchronous batch call; hull meshes cached under _build/meshes between runs."""
    from math_b200 import batched

    os.environ.setdefault("NTRACE_NO_BUILD", "1")
    r = batched.run(count=64, seed=0, repeat=args.steps, cache=ROOT / "_build" / "meshes")
    print(json.dumps({
        "metric": "paths/s (batched mixed workload, n = 3..6)", "value": r["batch_paths_per_s"], "unit": "paths/s",
        "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": 1000 * r["batch_seconds"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": r["workload"]}, "sequential_paths_per_s": r["sequential_paths_per_s"],
        "paths_per_pass": r["paths_per_pass"], "tuned": r["tuned"], "dims": r["dims"], "facets": r["facets"],
        "screens": r["screens"]}))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="n4")
    ap.add_argument("--cpu-paths", type=int, default=8_000_000, help="paths in the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other dimensions' lines and the denoised-versus-plain measurement")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        if args.config == "batch":
            print(json.dumps({"impl": "reference", "unavailable": "the batched mixed workload has no reference "
                              "counterpart (the reference paints one scene per paint() call)"}))
            return
        run_reference(args)
        return

    import torch

    if args.config == "batch":
        run_batch(args)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    os.environ.setdefault("NTRACE_NO_BUILD", "1")
    from math_b200 import scenes

    extras = rank == 0 and world == 1 and not args.no_extras
    others = [c for c in ("n3", "n4", "n5") if c != args.config] if extras else []
    # the other configurations' meshes (the n = 5 hull takes tens of seconds on the host) are prepared
    # on a host thread while the headline configuration runs on the GPU
    prepared: dict = {}

    def prepare():
        for c in others:
            prepared[c] = scenes.config(c)

    prep = threading.Thread(target=prepare, daemon=True)
    prep.start()

    spec = scenes.config(args.config)
    n = spec["n"]
    scene = scenes.build_scene(spec, tree_on_gpu=True)
    from math_b200 import ntrace

    probes = ntrace.probe_peaks()
    m = measure_plain(scene, spec, args, args.steps, rank, world, local, dist)
    timed, tuned = m["timed"], m["tuned"]

    result = {
        "metric": metric_name(n), "value": m["value"], "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(spec, args),
        "mesh": mesh_block(spec, "exact (nt_convex_hull)"),
        "tuning": {"pool_paths": tuned["pool_paths"], "graph_iterations": tuned["graph_iterations"],
                   "walk_chunk": tuned["walk_chunk"], "walk_small_leaf": tuned["walk_small_leaf"],
                   "tuned_by": "nt_autotune"},
        "e2e": m["e2e"],
        "gpu_launches": m["launches"],
        "roofline": roofline(n, timed, args.config, tuned["pool_paths"], probes),
        "probed_peaks": probes,
        "kernels_ms_per_frame": {"raygen": timed["raygen_ms"], "plan": timed["plan_ms"], "extend": timed["extend_ms"],
                                 "shade": timed["shade_ms"], "shadow": timed["shadow_ms"]},
        "counters_per_frame": {k: timed[k] for k in ("rays", "shadow_rays", "facet_tests", "box_steps", "retests",
                                                     "descent_levels", "shadow_facet_tests", "shadow_box_steps",
                                                     "shadow_retests", "shadow_descent_levels")},
        "clocks": m["clocks"],
        "device_errors": m["device_errors"],
    }
    if "combine_ms" in m:
        result["combine_ms"] = m["combine_ms"]
    if extras:
        # the other dimensions (fewer steps) and the denoised-versus-plain time to the target error
        denoise_res = {}
        try:
            denoise_res[args.config] = measure_denoise(scene, n)
        except Exception as e:  # report it; the headline line stands
            denoise_res[args.config] = {"error": repr(e)}
        scene.close()
        prep.join()
        per_n = {}
        for c in others:
            sp = prepared[c]
            sc = scenes.build_scene(sp, tree_on_gpu=True)
            k = min(args.steps, 5)
            mm = measure_plain(sc, sp, args, k, rank, world, local, dist)
            per_n[c] = {"metric": metric_name(sp["n"]), "value": mm["value"], "unit": "paths/s",
                        "ms_per_step": mm["ms_per_step"], "steps": k, "e2e": mm["e2e"],
                        "config": config_block(sp, argparse.Namespace(config=c)),
                        "mesh": mesh_block(sp, "exact (nt_convex_hull)"),
                        "tuning": {"pool_paths": mm["tuned"]["pool_paths"],
                                   "graph_iterations": mm["tuned"]["graph_iterations"],
                                   "walk_chunk": mm["tuned"]["walk_chunk"],
                                   "walk_small_leaf": mm["tuned"]["walk_small_leaf"]},
                        "roofline": roofline(sp["n"], mm["timed"], c, mm["tuned"]["pool_paths"], probes),
                        "kernels_ms_per_frame": {kk: mm["timed"][kk + "_ms"] for kk in ("raygen", "plan", "extend",
                                                                                        "shade", "shadow")},
                        "clocks": mm["clocks"], "device_errors": mm["device_errors"]}
            try:
                denoise_res[c] = measure_denoise(sc, sp["n"])
            except Exception as e:
                denoise_res[c] = {"error": repr(e)}
            sc.close()
        result["per_n"] = per_n
        result["denoise_time_to_rmse_1e-2"] = denoise_res
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(spec, args.cpu_paths, os.cpu_count() or 1)
        # the same painter on one thread, over an eighth of the sample
        one = cpu_baseline(spec, max(1000, args.cpu_paths // 8), 1)
        result["cpu_baseline"]["single_thread"] = {k: one[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        print(json.dumps(result))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
