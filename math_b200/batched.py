"""The batched mixed workload: many scenes of mixed dimension and size rendered side by side in one
CUDA graph (nt_render_batch), with per-dimension pool sizes and iterations per graph launch chosen by
the autotuner (nt_autotune).

    python -m math_b200.batched --scenes 64 --seed 0

Scenes: n uniform in {3, 4, 5, 6}; boundary of the convex hull of seeded points on the unit sphere,
point counts log-uniform in a per-dimension range; the floor, light and parallel camera of
the measured scenes; screens log-uniform per dimension; 1 to 16 samples per pixel.  Prints one JSON
line: paths/s of the batch, of the same passes rendered one after the other, and the tuned
parameters per n (pool size, iterations per graph launch, walk staging chunk).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time
from pathlib import Path

import numpy as np

from . import ntrace, scenes

# Per-dimension point-count ranges.  The configuration asks for [1e3, 2e5] at every n; the exact hull
# that makes the meshes runs on the host, and its time sets the upper ends at n = 5 and 6 (measured in
# this container: n = 4, 2e5 points, 1.35 M facets: 105 s; n = 5, 1e5 points, 3.1 M facets: 113 s;
# n = 6, 5e3 points, 0.78 M facets: 59 s; the facet count per point grows steeply with n, so a 2e5-point
# hull at n = 6 would hold some 2e7 facets and take hours).
POINT_RANGE = {3: (1_000, 200_000), 4: (1_000, 200_000), 5: (1_000, 50_000), 6: (1_000, 3_000)}
# path pool per scene at most (the batch's pools are resident together)
MAX_POOL = 16 << 20
# screens from 64^2 (n = 3) up to 32^5 (n = 6) pixels
SCREEN_RANGE = {3: (64, 512), 4: (32, 128), 5: (16, 48), 6: (8, 32)}


def scene_mesh(n: int, points: int, seed: int, cache: Path | None):
    """The hull mesh of one batch scene, from the on-disk cache when there is one."""
    if cache is not None:
        f = cache / f"hull_n{n}_p{points}_s{seed}.npz"
        if f.exists():
            z = np.load(f)
            return z["verts"], z["facets"]
    v, fc = scenes.sphere_hull(n, points, seed=seed)
    if cache is not None:
        cache.mkdir(parents=True, exist_ok=True)
        np.savez(cache / f"hull_n{n}_p{points}_s{seed}.npz", verts=v, facets=fc)
    return v, fc


def make_workload(count: int, seed: int, cache: Path | None = None, max_points: int | None = None) -> list[dict]:
    """`count` seeded scenes: n uniform in {3, 4, 5, 6}, point counts log-uniform in POINT_RANGE[n] (capped
    at max_points), screens log-uniform in SCREEN_RANGE[n], 1 to 16 samples per pixel."""
    rng = np.random.default_rng(seed)
    plans = []
    for i in range(count):
        n = int(rng.integers(3, 7))
        plo, phi = POINT_RANGE[n]
        points = int(round(math.exp(rng.uniform(math.log(plo), math.log(phi)))))
        if max_points:
            points = min(points, max_points)
        lo, hi = SCREEN_RANGE[n]
        screen = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        spp = int(rng.integers(1, 17))
        plans.append((n, points, screen, spp, i))
    # the hulls on host threads (the library's hull call releases the interpreter lock), largest first
    from concurrent.futures import ThreadPoolExecutor

    order = sorted(range(count), key=lambda k: -plans[k][1] * 2 ** plans[k][0])
    with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as ex:
        meshes = dict(zip(order, ex.map(lambda k: scene_mesh(plans[k][0], plans[k][1], seed * 1000 + plans[k][4], cache),
                                        order)))
    specs = []
    for k, (n, points, screen, spp, i) in enumerate(plans):
        v, f = meshes[k]
        spec = scenes.make_spec(n, v, f, screen=screen, spp=spp, max_depth=5, seed=i)
        spec["points"] = points
        specs.append(spec)
    return specs


def run(count: int = 64, seed: int = 0, repeat: int = 3, cache: Path | None = None,
        max_points: int | None = None) -> dict:
    """Builds the workload, tunes per dimension, and times the batch (one graph per pass of all scenes)
    against the same passes one after the other."""
    import torch

    t0 = time.perf_counter()
    specs = make_workload(count, seed, cache, max_points)
    mesh_s = time.perf_counter() - t0
    # the 64 scenes stay resident together, so their meshes keep only the compact record arrays (no
    # leaf-ordered copy, which repeats a record once per leaf listing it: several GB for the larger n = 5
    # and 6 hulls), and their path pools are capped at MAX_POOL paths
    built = [scenes.build_scene(sp, tree_on_gpu=True, leaf_records=-1) for sp in specs]
    build_s = time.perf_counter() - t0
    # autotune once per dimension on its largest scene; apply to every scene of that dimension
    tuned = {}
    for n in (3, 4, 5, 6):
        idx = [i for i, sp in enumerate(specs) if sp["n"] == n]
        if not idx:
            continue
        big = max(idx, key=lambda i: built[i].pixel_count * ntrace.effective_spp(n, specs[i]["spp"]))
        t, ms = built[big].autotune(specs[big]["spp"], max_depth=5)
        tuned[n] = dict(t, probe_ms=ms)
    opts = []
    for sp in specs:
        t = tuned[sp["n"]]
        opts.append(dict(samples_per_pixel=sp["spp"], max_depth=5, seed=sp["seed"],
                         pool_paths=min(t["pool_paths"], MAX_POOL),
                         graph_iterations=t["graph_iterations"], walk_chunk=t["walk_chunk"],
                         walk_small_leaf=t["walk_small_leaf"]))
    paths = sum(s.pixel_count * ntrace.effective_spp(sp["n"], sp["spp"]) for s, sp in zip(built, specs))
    # warm-up, then timed passes
    ntrace.render_batch(built, opts)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(repeat):
        ntrace.render_batch(built, opts)
    batch_s = (time.perf_counter() - t0) / repeat
    t0 = time.perf_counter()
    for _ in range(repeat):
        for s, o in zip(built, opts):
            s.render(**o)
    seq_s = (time.perf_counter() - t0) / repeat
    out = {
        "workload": f"{count} scenes, n in 3..6, hull meshes of {POINT_RANGE} points (capped at {max_points}), "
                    f"screens {SCREEN_RANGE} per axis, 1-16 spp",
        "scenes": count, "paths_per_pass": paths, "mesh_seconds": mesh_s, "build_seconds": build_s,
        "batch_paths_per_s": paths / batch_s, "sequential_paths_per_s": paths / seq_s, "batch_seconds": batch_s,
        "sequential_seconds": seq_s, "tuned": {str(k): v for k, v in tuned.items()},
        "facets": [int(len(sp["facets"])) for sp in specs], "points": [sp["points"] for sp in specs],
        "mesh_device_bytes": [int(s.mesh_info(0)["device_bytes"]) for s in built],
        "screens": [sp["projector"]["screen"][0] for sp in specs], "dims": [sp["n"] for sp in specs],
    }
    for sc in built:
        sc.close()
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--cache", default=None, help="directory for the generated hull meshes (reused across runs)")
    ap.add_argument("--max-points", type=int, default=None, help="cap on the point counts (quick runs)")
    args = ap.parse_args(argv)
    print(json.dumps(run(args.scenes, args.seed, args.repeat, Path(args.cache) if args.cache else None,
                         args.max_points)), flush=True)


if __name__ == "__main__":
    sys.exit(main())
