"""Generates the committed golden fixtures from the reference painter itself.

Run in a checkout where the reference sources are present (they are compiled in place by
oracle/Makefile into oracle/_ref/libref_painter.so):

    python tests/golden/make_golden.py

Fixtures (numpy .npz, small enough to commit):
  closest_n{3,4,5,6}.npz  - a seeded sphere mesh (vertices float32, facets int32), a seeded ray set
                            (org, dir float32) and the reference's closest hit for each ray through
                            Mesh<N,double> and Mesh<N,float> (facet index, -1 = miss; distance),
                            queried as src/painter/shapes/test/test_mesh.cpp:139-152 does; plus the
                            reference tree's box and index counts.
  radiance_n3.npz          - the reference's paint<3,double>() of a 24 x 24 floor scene at 1024 samples
                            per pixel, painted twice with different seeds (one thread, seeded engines),
                            so that a test can compare another renderer's image against the reference
                            with the reference's own run-to-run noise as the yardstick.
  radiance_n3_smooth.npz   - the same, the view closed in on the sphere (2.4 x 2.4), with vertex
                            normals of every NormalType and smooth_normal set (smooth_mesh below).
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from math_b200 import scenes  # noqa: E402
from oracle import checkers  # noqa: E402

OUT = Path(__file__).resolve().parent


def ray_set(n: int, count: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Rays from a sphere of radius 2 towards the centre, perturbed (test_mesh.cpp:46-67 style)."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((count, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = (2.0 * d + 0.0131).astype(np.float32)
    dirs = (-d + 0.08 * rng.standard_normal((count, n))).astype(np.float32)
    return org, dirs


def edge_rays(verts: np.ndarray, facets: np.ndarray, count: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Rays aimed from outside at points on facet boundaries (edge midpoints and vertices), where the
    barycentric decision is hardest and float and double disagree most often."""
    rng = np.random.default_rng(seed)
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
    org = target + 2.5 * d
    return org.astype(np.float32), (target - org).astype(np.float32)


CASES = {
    3: dict(mesh=lambda: scenes.icosphere(2), rays=4000),
    4: dict(mesh=lambda: scenes.sphere_hull(4, 300, seed=11), rays=3000),
    5: dict(mesh=lambda: scenes.sphere_hull(5, 80, seed=12), rays=2000),
    6: dict(mesh=lambda: scenes.sphere_hull(6, 30, seed=13), rays=1000),
}


def closest_fixtures(ref: checkers.Reference) -> None:
    for n, case in CASES.items():
        t0 = time.time()
        verts, facets = case["mesh"]()
        org, dirs = ray_set(n, case["rays"], seed=100 + n)
        eo, ed = edge_rays(verts, facets, case["rays"] // 2, seed=200 + n)
        org = np.concatenate([org, eo])
        dirs = np.concatenate([dirs, ed])
        m64 = ref.mesh(n, verts, facets, dbl=True)
        f64, t64 = ref.trace(m64, org, dirs)
        m32 = ref.mesh(n, verts, facets, dbl=False)
        f32, t32 = ref.trace(m32, org, dirs)
        i64 = ref.tree_info(m64)
        i32 = ref.tree_info(m32)
        np.savez_compressed(OUT / f"closest_n{n}.npz", verts=verts, facets=facets, org=org, dir=dirs, facet64=f64,
                            t64=t64, facet32=f32, t32=t32, boxes64=i64["box_count"], indices64=i64["index_count"],
                            boxes32=i32["box_count"], indices32=i32["index_count"])
        print(f"n={n}: {len(facets)} facets, {len(org)} rays, {(f64 < 0).sum()} misses, "
              f"{(f64 != f32).sum()} fp32/fp64 facet differences, {time.time() - t0:.1f}s")


def radiance_fixture(ref: checkers.Reference) -> None:
    verts, facets = scenes.icosphere(1)
    spec = scenes.make_spec(3, verts, facets, screen=24, spp=1024, max_depth=5)
    t0 = time.time()
    img_a, st_a = ref.paint(spec, dbl=True, seed=1, threads=1)
    img_b, st_b = ref.paint(spec, dbl=True, seed=2, threads=1)
    np.savez_compressed(OUT / "radiance_n3.npz", verts=verts, facets=facets, screen=24, spp=1024, max_depth=5,
                        image_a=img_a, image_b=img_b, samples=st_a["sample_count"])
    rr = np.sqrt(((img_a - img_b) ** 2).sum() / (img_b ** 2).sum())
    print(f"radiance: {img_a.shape}, run-to-run relative RMSE {rr:.4g}, {time.time() - t0:.1f}s")


def smooth_mesh(subdivisions: int = 2, seed: int = 5) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """An icosphere with vertex normals that exercise every NormalType of MeshHyperplaneSimplex
    (mesh_hyperplane_simplex.cpp:96-143): sphere normals (Use), every 5th facet wound backwards (all
    vertex normals opposite the facet normal: Use with the facet normal reversed), every 11th vertex
    normal negated (mixed signs: Reverse), every 13th vertex normal tilted by 60 degrees (|cos| < 0.7:
    None)."""
    rng = np.random.default_rng(seed)
    verts, facets = scenes.icosphere(subdivisions)
    normals = verts / np.linalg.norm(verts, axis=1, keepdims=True)
    facets = facets.copy()
    facets[::5, [0, 1]] = facets[::5, [1, 0]]
    normals[::11] *= -1
    for i in range(0, len(normals), 13):
        t = rng.standard_normal(3)
        t -= np.dot(t, normals[i]) * normals[i]
        t /= np.linalg.norm(t)
        normals[i] = 0.5 * normals[i] + np.sqrt(0.75) * t
    return verts.astype(np.float32), facets.astype(np.int32), normals.astype(np.float32)


def radiance_smooth_fixture(ref: checkers.Reference) -> None:
    verts, facets, normals = smooth_mesh()
    spec = scenes.make_spec(3, verts, facets, screen=24, spp=1024, max_depth=5, extent=2.4)
    spec["normals"] = normals
    spec["smooth_normal"] = True
    t0 = time.time()
    img_a, st_a = ref.paint(spec, dbl=True, seed=1, threads=8)
    img_b, st_b = ref.paint(spec, dbl=True, seed=2, threads=8)
    np.savez_compressed(OUT / "radiance_n3_smooth.npz", verts=verts, facets=facets, normals=normals, screen=24,
                        extent=2.4, spp=1024, max_depth=5, image_a=img_a, image_b=img_b,
                        samples=st_a["sample_count"])
    rr = np.sqrt(((img_a - img_b) ** 2).sum() / (img_b ** 2).sum())
    print(f"radiance (smooth normals): {img_a.shape}, run-to-run relative RMSE {rr:.4g}, {time.time() - t0:.1f}s")


if __name__ == "__main__":
    checkers.build()
    reference = checkers.Reference()
    if "--smooth-only" not in sys.argv:
        closest_fixtures(reference)
        radiance_fixture(reference)
    radiance_smooth_fixture(reference)
