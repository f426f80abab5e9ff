"""The batched mixed workload: many scenes of mixed dimension and size rendered side by side in one
CUDA graph (nt_render_batch), with per-dimension pool sizes and iterations per graph launch chosen by
the autotuner (nt_autotune).

    python -m math_b200.batched --scenes 64 --seed 0

Scenes: n uniform in {3, 4, 5, 6}; boundary of the convex hull of seeded points on the unit sphere,
point counts log-uniform in a per-dimension range; the floor, light and parallel camera of
the measured scenes; screens log-uniform per dimension; 1 to 16 samples per pixel.  Prints one JSON
line: paths/s of the batch, of the same passes rendered one after the other, and the tuned
parameters per n.
"""

from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import ntrace, scenes

# per-dimension point-count ranges: hull size grows steeply with n, and the trees are built on the host
POINT_RANGE = {3: (1_000, 200_000), 4: (1_000, 20_000), 5: (500, 3_000), 6: (300, 800)}
SCREEN_RANGE = {3: (64, 256), 4: (32, 64), 5: (16, 32), 6: (8, 16)}


def make_workload(count: int, seed: int) -> list[dict]:
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(rng.integers(3, 7))
        plo, phi = POINT_RANGE[n]
        points = int(round(math.exp(rng.uniform(math.log(plo), math.log(phi)))))
        lo, hi = SCREEN_RANGE[n]
        screen = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        spp = int(rng.integers(1, 17))
        v, f = scenes.sphere_hull(n, points, seed=seed * 1000 + i)
        spec = scenes.make_spec(n, v, f, screen=screen, spp=spp, max_depth=5, seed=i)
        spec["points"] = points
        specs.append(spec)
    return specs


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args(argv)
    import torch

    t0 = time.perf_counter()
    specs = make_workload(args.scenes, args.seed)
    built = [scenes.build_scene(sp, tree_on_gpu=True) for sp in specs]
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
        opts.append(dict(samples_per_pixel=sp["spp"], max_depth=5, seed=sp["seed"], pool_paths=t["pool_paths"],
                         graph_iterations=t["graph_iterations"], walk_chunk=t["walk_chunk"]))
    paths = sum(s.pixel_count * ntrace.effective_spp(sp["n"], sp["spp"]) for s, sp in zip(built, specs))
    # warm-up, then timed passes
    ntrace.render_batch(built, opts)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.repeat):
        ntrace.render_batch(built, opts)
    batch_s = (time.perf_counter() - t0) / args.repeat
    t0 = time.perf_counter()
    for _ in range(args.repeat):
        for s, o in zip(built, opts):
            s.render(**o)
    seq_s = (time.perf_counter() - t0) / args.repeat
    print(json.dumps({
        "workload": f"{args.scenes} scenes, n in 3..6, hull meshes of {POINT_RANGE} points, screens {SCREEN_RANGE}, 1-16 spp",
        "scenes": args.scenes, "paths_per_pass": paths, "build_seconds": build_s,
        "batch_paths_per_s": paths / batch_s, "sequential_paths_per_s": paths / seq_s, "batch_seconds": batch_s,
        "sequential_seconds": seq_s, "tuned": {str(k): v for k, v in tuned.items()},
        "facets": [int(len(sp["facets"])) for sp in specs], "dims": [sp["n"] for sp in specs],
    }), flush=True)


if __name__ == "__main__":
    sys.exit(main())
