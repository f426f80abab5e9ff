"""Trains the learned denoiser (one network per dimension) on pairs rendered by the tracer, and
measures the time to a relative RMSE of 1e-2 against a 64k-sample render, plain versus denoised.

    python -m math_b200.train_denoiser --n 3 4 5 --pairs 200 --steps 3000 --out math_b200/weights

Training pairs: seeded variations (light position, view direction, albedos in [0.3, 0.9]) of the
measured scenes' meshes on small screens; the noisy input is a few samples per pixel (its per-pixel
mean and variance of the mean), plus the first-hit normal and depth; the target is a 4096-sample
render.  The input sample count of each pair is k^(n-1) (a full stratification grid, k per screen
axis) with k drawn from --k-in, so one network covers several noise levels.  Weights go to
<out>/denoiser_n<n>.npz.

Evaluation (--eval): a held-out variation at the measured configuration's screen size (400^2, 128^3,
48^4); plain and denoised renders on the same sample grid, k^(n-1) samples for k = 1, 2, 3, ...,
timed over the whole frame, give (time, relative RMSE) points, the error measured on the centred
window (128^2, 32^3, 16^4) against a 64k-sample render of that window (effective k^(n-1) >= 65536);
the report is the time each method needs to reach --target (its first grid point at or below it),
and the plain time fitted to the target exactly (Monte Carlo error ~ 1/sqrt(spp), time ~ spp).
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import denoise, ntrace, scenes

TRAIN_SCREEN = {3: 64, 4: 24, 5: 10, 6: 6}    # training crops, at the measured screen's pixel scale
EVAL_SCREEN = {3: 400, 4: 128, 5: 48, 6: 16}   # the measured configurations' screens over the 8 x ... x 8 view
REF_CROP = {3: 128, 4: 32, 5: 16, 6: 8}        # centred window rendered at 64k samples as the reference
EXTENT = 8.0
CROP_EXTENT = 4.0                              # training crops lie inside the central 4 x ... x 4 region
REF_SPP = 65536


def mesh_for(n: int, small: bool = False):
    """The measured scene's mesh (or the reduced test mesh)."""
    if small:
        return scenes.config(f"n{n}_small")
    if n == 3:
        v, f = scenes.icosphere(5)
        return scenes.make_spec(3, v, f, screen=TRAIN_SCREEN[3], spp=4)
    if n == 4:
        v, f = scenes.sphere_hull(4, 100_000, seed=0)
        return scenes.make_spec(4, v, f, screen=TRAIN_SCREEN[4], spp=4)
    if n == 5:
        v, f = scenes.sphere_hull(5, 50_000, seed=0, cap=0.5)
        return scenes.make_spec(5, v, f, screen=TRAIN_SCREEN[5], spp=4)
    v, f = scenes.sphere_hull(6, 5_000, seed=0)
    return scenes.make_spec(6, v, f, screen=TRAIN_SCREEN[6], spp=4)


def make_mixed_pairs(scene, n: int, count: int, seed: int, k_in: list[int], spp_ref: int) -> list[dict]:
    pairs = []
    rng = np.random.default_rng(seed)
    for i in range(count):
        s = int(k_in[rng.integers(len(k_in))]) ** (n - 1)
        pairs += denoise.make_pairs(scene, 1, seed=seed * 7919 + i, screen=TRAIN_SCREEN[n], spp_in=s, spp_ref=spp_ref,
                                    units_per_pixel=EXTENT / EVAL_SCREEN[n], extent=CROP_EXTENT)
    return pairs


def crop(img, n: int, full: int, size: int):
    """The centred size^(n-1) window of a full^(n-1) image (pixels x0 fastest)."""
    a = np.asarray(img.detach().cpu() if hasattr(img, "detach") else img).reshape([full] * (n - 1) + [3])
    o = (full - size) // 2
    return a[tuple([slice(o, o + size)] * (n - 1))].reshape(-1, 3)


def time_to_rmse(scene, den, n: int, target: float, seed: int, max_plain_spp: int = 1 << 12) -> dict:
    """Plain and denoised renders of one held-out variation at the measured screen size, timed over
    the whole frame, at k^(n-1) samples for k = 1, 2, ... until each reaches the target; their error
    is measured on the centred window against a 64k-sample render of that window (same pixel
    grid)."""
    import torch

    full, size = EVAL_SCREEN[n], REF_CROP[n]
    rng = np.random.default_rng(seed)
    v = denoise.random_variant(n, rng, full)
    w = dict(v, screen=[size] * (n - 1))
    denoise.apply_variant(scene, w)
    t0 = time.perf_counter()
    ref = denoise.render_reference(scene, REF_SPP, seed=seed + 1).cpu().numpy()
    ref_s = time.perf_counter() - t0
    denoise.apply_variant(scene, v)
    plain = []
    k = 1
    while k ** (n - 1) <= max_plain_spp:
        spp = k ** (n - 1)
        # warm (graphs and pools of this sample count), then timed
        scene.clear()
        scene.render(spp, max_depth=5, seed=seed + 3 + spp)
        scene.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scene.render(spp, max_depth=5, seed=seed + 2 + spp)
        dt = time.perf_counter() - t0
        img, _ = scene.image()
        plain.append({"spp": ntrace.effective_spp(n, spp), "seconds": dt,
                      "rmse": denoise.relative_rmse(crop(img, n, full, size), ref)})
        if plain[-1]["rmse"] <= target:
            break
        k += 1
    den_pts = []
    k = 1
    while k ** (n - 1) <= max_plain_spp:
        s = k ** (n - 1)
        k += 1
        # warm (the denoiser's workspace is allocated on first use)
        x = denoise.render_inputs(scene, s, seed=seed + 5)
        den.set_input(v["screen"], x["mean"], x["var"], x["normal"], x["depth"], s)
        den.apply()
        torch.cuda.synchronize()
        parts = {}
        t0 = time.perf_counter()
        x = denoise.render_inputs(scene, s, seed=seed + 7, timing=parts)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        den.set_input(v["screen"], x["mean"], x["var"], x["normal"], x["depth"], s)
        out = den.apply()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        den_pts.append({"spp": ntrace.effective_spp(n, s), "seconds": t2 - t0, "render_seconds": t1 - t0,
                        "network_seconds": t2 - t1, **parts,
                        "rmse": denoise.relative_rmse(crop(out, n, full, size), ref),
                        "input_rmse": denoise.relative_rmse(crop(x["mean"], n, full, size), ref)})
        if den_pts[-1]["rmse"] <= target:
            break

    def first(points):
        ok = [p for p in points if p["rmse"] <= target]
        return min(ok, key=lambda p: p["seconds"]) if ok else None

    bp, bd = first(plain), first(den_pts)
    # plain Monte Carlo error falls as 1/sqrt(spp) and its time grows as spp: the plain time at exactly
    # the target, from its last grid point (the interpolation favours the plain render)
    last = plain[-1]
    plain_fit = last["seconds"] * (last["rmse"] / target) ** 2
    return {"n": n, "screen": [full] * (n - 1), "reference_window": [size] * (n - 1),
            "reference_spp": ntrace.effective_spp(n, REF_SPP), "reference_seconds": ref_s, "target_rmse": target,
            "plain": plain, "denoised": den_pts,
            "plain_time_to_target": bp["seconds"] if bp else None,
            "denoised_time_to_target": bd["seconds"] if bd else None,
            "speedup": (bp["seconds"] / bd["seconds"]) if (bp and bd) else None,
            "plain_time_to_target_fitted": plain_fit,
            "speedup_vs_fitted": (plain_fit / bd["seconds"]) if bd else None}


def synthetic(args) -> None:
    """Training steps on seeded random features (square-ish screen of about --synthetic pixels): the
    throughput of the network's kernels alone."""
    import torch

    for n in args.n:
        side = max(4, int(round(args.synthetic ** (1.0 / (n - 1)))))
        screen = [side] * (n - 1)
        P = side ** (n - 1)
        g = torch.Generator(device="cpu").manual_seed(args.seed + n)
        mean = torch.rand(P, 3, generator=g).cuda()
        var = (torch.rand(P, 3, generator=g) * 0.01).cuda()
        normal = torch.nn.functional.normalize(torch.randn(P, n, generator=g), dim=1).cuda()
        depth = (torch.rand(P, generator=g) * 5 + 5).cuda()
        target = (mean + 0.05 * torch.randn(P, 3, generator=g).cuda()).clamp_min(0).contiguous()
        den = denoise.Denoiser(n, seed=args.seed)
        den.set_input(screen, mean, var, normal, depth, 4)
        den.train_step(target, args.lr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            den.train_step(target, args.lr)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / max(1, args.steps)
        t0 = time.perf_counter()
        den.apply()
        torch.cuda.synchronize()
        fwd = time.perf_counter() - t0
        L = den.layout
        flops = 2 * P * (L["features_padded"] * L["hidden"] + L["hidden"] * L["hidden"] + L["hidden"] * L["outputs_padded"])
        print(json.dumps({"n": n, "pixels": P, "train_step_ms": dt * 1e3, "apply_ms": fwd * 1e3,
                          "forward_gemm_tflops_per_s": flops / fwd / 1e12}), flush=True)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--n", type=int, nargs="+", default=[3, 4, 5])
    ap.add_argument("--pairs", type=int, default=200)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=None,
                    help="fall from --lr to this along a half cosine over the steps (default: constant --lr)")
    ap.add_argument("--k-in", type=int, nargs="+", default=[1, 2, 3, 4, 6, 8],
                    help="input samples per pixel of the training pairs: k^(n-1) for k drawn from these "
                         "(those with k^(n-1) above spp-ref / 16 are left out)")
    ap.add_argument("--spp-ref", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "weights"))
    ap.add_argument("--small", action="store_true", help="reduced test meshes instead of the measured ones")
    ap.add_argument("--eval", action="store_true")
    ap.add_argument("--target", type=float, default=1e-2)
    ap.add_argument("--load", action="store_true", help="evaluate saved weights instead of training")
    ap.add_argument("--synthetic", type=int, default=0,
                    help="train on seeded synthetic inputs of this many pixels (kernel throughput; no rendering)")
    args = ap.parse_args(argv)
    if args.synthetic:
        synthetic(args)
        return
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for n in args.n:
        k_in = [k for k in args.k_in if 16 * k ** (n - 1) <= args.spp_ref] or [1]
        t0 = time.perf_counter()
        spec = mesh_for(n, args.small)
        scene = scenes.build_scene(spec, tree_on_gpu=True)
        build_s = time.perf_counter() - t0
        path = out / f"denoiser_n{n}.npz"
        report = {"n": n, "scene_build_seconds": build_s, "k_in": k_in, "pairs": args.pairs, "steps": args.steps,
                  "lr": args.lr, "lr_final": args.lr_final}
        if args.load:
            den = denoise.Denoiser.load(path)
        else:
            t0 = time.perf_counter()
            pairs = make_mixed_pairs(scene, n, args.pairs, args.seed + n, k_in, args.spp_ref)
            report["pairs_seconds"] = time.perf_counter() - t0
            held = make_mixed_pairs(scene, n, max(4, args.pairs // 10), args.seed + 1000 + n, k_in,
                                    args.spp_ref)
            den = denoise.Denoiser(n, seed=args.seed)
            uni = denoise.Denoiser(n, seed=args.seed)
            uni.set_params(denoise.uniform_filter_params(uni))
            t0 = time.perf_counter()
            losses = denoise.train(den, pairs, args.steps, args.lr, seed=args.seed, lr_final=args.lr_final)
            report["train_seconds"] = time.perf_counter() - t0
            report["loss_first_100"] = float(np.mean(losses[:100]))
            report["loss_last_100"] = float(np.mean(losses[-100:]))
            report["held_out"] = {"trained": denoise.evaluate(den, held), "uniform": denoise.evaluate(uni, held)}
            den.save(path)
            report["weights"] = str(path)
        if args.eval:
            report["time_to_rmse"] = time_to_rmse(scene, den, n, args.target, seed=args.seed + 77 + n)
        print(json.dumps(report), flush=True)
        scene.close()


if __name__ == "__main__":
    sys.exit(main())
