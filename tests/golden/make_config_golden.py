"""Generates the committed configuration-scale fixtures from the reference painter itself.

Run in a checkout where the reference sources are present (they are compiled in place by
oracle/Makefile into oracle/_ref/libref_painter.so):

    python tests/golden/make_config_golden.py [--rays] [--radiance] [--images] [name ...]

The meshes are not stored: each fixture records the facet and vertex counts and a SHA-256 of the
float32 vertex and int32 facet arrays that math_b200.scenes produces for its configuration (seeded
points, the library's exact convex hull), and the tests rebuild the mesh and check those first.

Fixtures (numpy .npz):
  config_rays_{n3,n4,n5}.npz   - 12,000 rays through the measured meshes (20,480 / 675,461 /
        1,541,774 facets) and the reference's closest hit of each through Mesh<N,double>
        (facet index, -1 = miss; distance), queried as src/painter/shapes/test/test_mesh.cpp:139-152:
        4,000 camera rays of random pixels (jittered, the configuration's parallel projector; half of
        them over the mesh), 4,000
        rays leaving the floor's top face upwards in random directions and 2,000 shadow rays from the
        same floor points to the light (the secondary and shadow rays of the paths under the mesh), and
        2,000 rays aimed from outside at facet edge midpoints and vertices.
  config_radiance_{n3,n4,n5,n6}.npz - 1,024 seeded pixels of the configuration scene (n6: the
        six-dimensional scene of math_b200.scenes.config("n6")) painted by the reference's
        paint<N,double>() at 65,536 samples per pixel (the reference rounds to k^(n-1): 65,536 at
        n = 3 and 5, 68,921 at n = 4, 100,000 at n = 6) twice, with different seeds, through a
        Paintbrush that hands out the pixel list (src/painter/painter.cpp:410-448).
  radiance_{n4,n5,n6}_small.npz - whole images of the small n = 4, 5, 6 scenes (12^3, 6^4, 4^5
        pixels) painted by paint<N,double>() at 1,024 samples per pixel (1,331 / 1,296 / 1,024
        effective), twice with different seeds.
  radiance_iface_*.npz - the same for the scenes of math_b200.scenes.interface_scene (ConstantLight,
        perspective and spherical projectors, a hyperplane parallelotope, two meshes).
"""

from __future__ import annotations

import hashlib
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from math_b200 import scenes  # noqa: E402
from oracle import checkers  # noqa: E402

OUT = Path(__file__).resolve().parent
THREADS = os.cpu_count() or 1


def mesh_digest(verts: np.ndarray, facets: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(verts, np.float32).tobytes())
    h.update(np.ascontiguousarray(facets, np.int32).tobytes())
    return h.hexdigest()


def random_pixels(screen, count: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    total = int(np.prod(screen))
    lin = np.sort(rng.choice(total, count, replace=False))
    return np.stack([(lin // int(np.prod(screen[:j]))) % screen[j] for j in range(len(screen))], axis=1).astype(np.int32)


def camera_rays(spec: dict, count: int, rng) -> tuple[np.ndarray, np.ndarray]:
    """Parallel-projector rays (projector.h:153-202) of random pixels with a uniform jitter."""
    P = spec["projector"]
    n = spec["n"]
    screen = np.asarray(P["screen"])
    axes = np.asarray(P["axes"], np.float64)
    axes = axes / np.linalg.norm(axes, axis=1, keepdims=True) * P["param"]
    point = rng.integers(0, screen, (count, n - 1)) + rng.random((count, n - 1)) - screen / 2.0
    # half of them in the pixels over the unit sphere's shadow on the screen
    half = count // 2
    point[:half] = rng.uniform(-1.1, 1.1, (half, n - 1)) / P["param"]
    org = np.asarray(P["org"], np.float64) + point @ axes
    d = np.broadcast_to(np.asarray(P["dir"], np.float64), org.shape)
    return org.astype(np.float32), np.ascontiguousarray(d, np.float32)


def floor_points(spec: dict, count: int, rng) -> np.ndarray:
    """Points on the floor slab's top face (last coordinate -1) under and around the mesh."""
    n = spec["n"]
    p = np.empty((count, n))
    p[:, : n - 1] = rng.uniform(-2.0, 2.0, (count, n - 1))
    p[:, n - 1] = -1.0 + 4.8e-4  # the tracer's ray offset above the face
    return p


def edge_rays(verts: np.ndarray, facets: np.ndarray, count: int, rng) -> tuple[np.ndarray, np.ndarray]:
    n = verts.shape[1]
    fi = rng.integers(0, len(facets), count)
    a = rng.integers(0, n, count)
    b = (a + rng.integers(1, n, count)) % n
    va = verts[facets[fi, a]].astype(np.float64)
    vb = verts[facets[fi, b]].astype(np.float64)
    w = np.where(rng.random(count) < 0.5, 0.5, 0.0)[:, None]
    target = va * (1 - w) + vb * w
    d = rng.standard_normal((count, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:, n - 1] = np.abs(d[:, n - 1])  # from above: the cap hole of the n = 5 mesh lets some in
    org = target + 2.5 * d
    return org.astype(np.float32), (target - org).astype(np.float32)


def config_ray_set(spec: dict, seed: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    n = spec["n"]
    co, cd = camera_rays(spec, 4000, rng)
    fp = floor_points(spec, 4000, rng)
    up = rng.standard_normal((4000, n))
    up /= np.linalg.norm(up, axis=1, keepdims=True)
    up[:, n - 1] = np.abs(up[:, n - 1]) + 0.05
    light = np.asarray(spec["light"]["pos"], np.float64)
    so = fp[:2000]
    sd = light - so
    eo, ed = edge_rays(spec["verts"], spec["facets"], 2000, rng)
    org = np.concatenate([co, fp.astype(np.float32), so.astype(np.float32), eo])
    dirs = np.concatenate([cd, up.astype(np.float32), sd.astype(np.float32), ed])
    kind = np.concatenate([np.full(4000, 0), np.full(4000, 1), np.full(2000, 2), np.full(2000, 3)]).astype(np.int8)
    return org, dirs, kind


def rays_fixture(ref: checkers.Reference, name: str) -> None:
    t0 = time.time()
    spec = scenes.config(name)
    n = spec["n"]
    verts, facets = spec["verts"], spec["facets"]
    org, dirs, kind = config_ray_set(spec, seed=300 + n)
    m64 = ref.mesh(n, verts, facets, dbl=True, threads=THREADS)
    t1 = time.time()
    f64, t64 = ref.trace(m64, org, dirs)
    info = ref.tree_info(m64)
    np.savez_compressed(OUT / f"config_rays_{name}.npz", org=org, dir=dirs, kind=kind, facet64=f64, t64=t64,
                        facet_count=len(facets), vertex_count=len(verts), digest=mesh_digest(verts, facets),
                        boxes64=info["box_count"], indices64=info["index_count"])
    print(f"{name}: {len(facets)} facets, Mesh<{n},double> built in {t1 - t0:.1f}s, {len(org)} rays, "
          f"{(f64 >= 0).sum()} hits ({[(int(((f64 >= 0) & (kind == k)).sum())) for k in range(4)]} by kind), "
          f"{time.time() - t0:.1f}s", flush=True)


RADIANCE_SPP = 65536


def radiance_fixture(ref: checkers.Reference, name: str, count: int = 1024) -> None:
    t0 = time.time()
    spec = scenes.config(name)
    n = spec["n"]
    px = random_pixels(spec["projector"]["screen"], count, seed=400 + n)
    img_a, st_a = ref.paint(spec, dbl=True, spp=RADIANCE_SPP, seed=11, threads=THREADS, pixels=px)
    img_b, st_b = ref.paint(spec, dbl=True, spp=RADIANCE_SPP, seed=9011, threads=THREADS, pixels=px)
    spp_eff = st_a["sample_count"] // count
    verts, facets = spec["verts"], spec["facets"]
    np.savez_compressed(OUT / f"config_radiance_{name}.npz", pixels=px, spp=RADIANCE_SPP, spp_effective=spp_eff,
                        max_depth=spec["max_depth"], image_a=img_a, image_b=img_b, facet_count=len(facets),
                        vertex_count=len(verts), digest=mesh_digest(verts, facets))
    rr = np.sqrt(((img_a - img_b) ** 2).sum() / (img_b ** 2).sum())
    print(f"{name}: {count} pixels x {spp_eff} spp twice, run-to-run relative RMSE {rr:.3g}, "
          f"{st_a['sample_count'] / st_a['seconds'] / 1e6:.2f} M paths/s, {time.time() - t0:.1f}s", flush=True)


def image_fixture(ref: checkers.Reference, name: str, spp: int = 1024) -> None:
    t0 = time.time()
    spec = scenes.config(name)
    img_a, st_a = ref.paint(spec, dbl=True, spp=spp, seed=21, threads=THREADS)
    img_b, _ = ref.paint(spec, dbl=True, spp=spp, seed=8021, threads=THREADS)
    verts, facets = spec["verts"], spec["facets"]
    np.savez_compressed(OUT / f"radiance_{name}.npz", spp=spp, max_depth=spec["max_depth"], image_a=img_a,
                        image_b=img_b, samples=st_a["sample_count"], facet_count=len(facets),
                        vertex_count=len(verts), digest=mesh_digest(verts, facets))
    rr = np.sqrt(((img_a - img_b) ** 2).sum() / (img_b ** 2).sum())
    print(f"{name}: {img_a.shape[0]} pixels x {spp} spp twice, run-to-run relative RMSE {rr:.3g}, "
          f"{time.time() - t0:.1f}s", flush=True)


def interface_fixture(ref: checkers.Reference, name: str, spp: int = 1024) -> None:
    t0 = time.time()
    spec = scenes.interface_scene(name)
    img_a, st_a = ref.paint(spec, dbl=True, spp=spp, seed=31, threads=THREADS)
    img_b, _ = ref.paint(spec, dbl=True, spp=spp, seed=8031, threads=THREADS)
    verts, facets = spec["verts"], spec["facets"]
    np.savez_compressed(OUT / f"radiance_iface_{name}.npz", spp=spp, max_depth=spec["max_depth"], image_a=img_a,
                        image_b=img_b, samples=st_a["sample_count"], facet_count=len(facets),
                        vertex_count=len(verts), digest=mesh_digest(verts, facets))
    rr = np.sqrt(((img_a - img_b) ** 2).sum() / (img_b ** 2).sum())
    print(f"{name}: {img_a.shape[0]} pixels x {spp} spp twice, run-to-run relative RMSE {rr:.3g}, "
          f"{time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    checkers.build()
    reference = checkers.Reference()
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    flags = {a for a in sys.argv[1:] if a.startswith("--")} or {"--rays", "--radiance", "--images", "--interface"}
    if "--rays" in flags:
        for nm in args or ["n3", "n4", "n5"]:
            rays_fixture(reference, nm)
    if "--radiance" in flags:
        for nm in args or ["n3", "n4", "n5", "n6"]:
            radiance_fixture(reference, nm)
    if "--images" in flags:
        for nm in args or ["n4_small", "n5_small", "n6_small"]:
            image_fixture(reference, nm)
    if "--interface" in flags:
        for nm in args or scenes.INTERFACE_SCENES:
            interface_fixture(reference, nm)
