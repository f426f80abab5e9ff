"""Renders whole frames of a configuration scene, for kernel profiles and launch lists.

    python -m math_b200.frame --config n4 [--pool 33554432] [--iterations 8] [--frames 2] [--stats]

The scene (`scenes.config`) is built with its trees on the GPU, then `--frames` frames of the
configuration's sample count are rendered with the given pool size and iterations per graph launch
(the walk variant and small-leaf threshold are the library's defaults unless given).  With --stats the
last frame is rendered with timing on, and its work counters and per-kernel event times are printed as
one JSON line.  A profiler run over this command sees the tree build first (k_overlap, k_write,
k_gather_records), then the frames' kernels in launch order: the first frame warms the graphs, so a
capture of the second frame's launches (skip the first frame's with the profiler's launch skip) shows
the steady state.
"""

from __future__ import annotations

import argparse
import json

from . import scenes

STAT_KEYS = ("paths", "iterations", "launches", "rays", "shadow_rays", "facet_tests", "box_steps", "descent_levels",
             "shadow_facet_tests", "shadow_box_steps", "shadow_descent_levels", "extend_launches", "shadow_launches",
             "raygen_ms", "plan_ms", "extend_ms", "shade_ms", "shadow_ms")


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--config", default="n4", help="a scenes.config name (n3, n4, n5, n6, n4_small, ...)")
    ap.add_argument("--pool", type=int, default=1 << 25, help="paths in flight (pool_paths)")
    ap.add_argument("--iterations", type=int, default=8, help="wavefront iterations per graph launch")
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--walk-chunk", type=int, default=0)
    ap.add_argument("--walk-small-leaf", type=int, default=0)
    ap.add_argument("--stats", action="store_true", help="time the last frame and print its counters")
    args = ap.parse_args(argv)
    spec = scenes.config(args.config)
    scene = scenes.build_scene(spec, tree_on_gpu=True)
    opts = dict(max_depth=5, seed=0, pool_paths=args.pool, graph_iterations=args.iterations,
                walk_chunk=args.walk_chunk, walk_small_leaf=args.walk_small_leaf)
    st = None
    for f in range(args.frames):
        st = scene.render(spec["spp"], **opts, timing=args.stats and f == args.frames - 1)
    if args.stats and st is not None:
        print(json.dumps({k: st[k] for k in STAT_KEYS if k in st} | {"config": args.config, "pool_paths": args.pool}))
    scene.close()


if __name__ == "__main__":
    main()
