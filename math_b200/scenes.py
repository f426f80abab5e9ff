"""Scene preparation: the meshes and scenes the path tracer is measured and checked on.

Mirrors the role of the reference's src/painter/scenes (single_object_scene,
src/painter/scenes/single_object.h:102-179): a mesh of (n-1)-simplices plus, here, a floor
parallelotope and a point light, seen through a parallel projector looking down the last axis.

Meshes:
  * ``icosphere(k)``: the icosahedron subdivided k times with vertices projected to the unit sphere
    (k = 5 gives 20,480 triangles).
  * ``sphere_hull(n, count, seed, cap)``: the boundary of the convex hull of ``count`` seeded points
    uniform on the unit (n-1)-sphere (normalised Gaussian vectors, numpy PCG64 seeded with ``seed``),
    optionally without the facets whose centroid lies within angular radius ``cap`` of +x_(n-1).  The
    hull is the library's exact convex hull (``nt_convex_hull``) of the float32 points, so every facet
    references exactly the vertices the tracer uses; ``method="qhull"`` takes scipy's Qhull instead,
    which gives the same facet set in another order (for processes that must not load the library).

A scene is a plain dict (``spec``) so that the same description feeds the product
(:func:`build_scene`) and the checkers in ``oracle/``.  Objects are added in the order mesh, second
mesh (``spec["mesh2"]``), floor parallelotope, hyperplane parallelotope (``spec["hplt"]``).
"""

from __future__ import annotations

import math

import numpy as np

from . import ntrace

# Background: emissive, as single_object_scene's default surface (single_object.h:71-74): colour
# for camera rays, a grey light of the colour's luminance for diffuse bounces.
BACKGROUND = (0.30, 0.35, 0.40)
BACKGROUND_LIGHT = (0.343, 0.343, 0.343)
ALBEDO = 0.7
# projector kinds (NT_PROJECTOR_*, include/ntrace.h)
PARALLEL, PERSPECTIVE, SPHERICAL = 0, 1, 2


def icosphere(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in verts]
    cache: dict[tuple[int, int], int] = {}

    def mid(a: int, b: int) -> int:
        key = (min(a, b), max(a, b))
        if key not in cache:
            m = (v[a] + v[b]) / 2.0
            v.append(m / np.linalg.norm(m))
            cache[key] = len(v) - 1
        return cache[key]

    for _ in range(subdivisions):
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(v, dtype=np.float32), np.array(faces, dtype=np.int32)


def sphere_points(n: int, count: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((count, n))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    return p.astype(np.float32)


def sphere_hull(n: int, count: int, seed: int, cap: float | None = None,
                method: str = "ntrace") -> tuple[np.ndarray, np.ndarray]:
    """Boundary of the convex hull of `count` seeded points on the unit (n-1)-sphere (the library's
    exact hull, nt_convex_hull; method="qhull": scipy's Qhull), optionally without the facets whose
    centroid direction lies within angle `cap` of +x_(n-1)."""
    pts = sphere_points(n, count, seed)
    if method == "qhull":
        from scipy.spatial import ConvexHull

        facets = ConvexHull(pts.astype(np.float64)).simplices.astype(np.int32)
    else:
        facets = ntrace.convex_hull(pts)
    if cap is not None:
        centroid = pts[facets].astype(np.float64).mean(axis=1)
        centroid /= np.linalg.norm(centroid, axis=1, keepdims=True)
        keep = centroid[:, n - 1] < math.cos(cap)
        facets = facets[keep]
    used = np.unique(facets)
    remap = np.full(len(pts), -1, np.int32)
    remap[used] = np.arange(len(used), dtype=np.int32)
    return np.ascontiguousarray(pts[used]), np.ascontiguousarray(remap[facets])


def floor_slab(n: int) -> tuple[np.ndarray, np.ndarray]:
    """[-4,4]^(n-1) x [-1.1,-1]."""
    org = np.full(n, -4.0, np.float32)
    org[n - 1] = -1.1
    edges = np.diag(np.full(n, 8.0, np.float32))
    edges[n - 1, n - 1] = 0.1
    return org, edges.astype(np.float32)


def make_spec(n: int, verts: np.ndarray | None, facets: np.ndarray | None, screen: int, spp: int, max_depth: int = 5,
              seed: int = 0, floor: bool = True, extent: float = 8.0, light_kind: int = 0,
              projector: int = 0) -> dict:
    """A floor scene: mesh, floor slab, one light at (2, ..., 2, 3), parallel projection of
    [-extent/2, extent/2]^(n-1) seen from +x_(n-1)."""
    light = np.full(n, 2.0, np.float32)
    light[n - 1] = 3.0
    cam = np.zeros(n, np.float32)
    cam[n - 1] = 10.0
    cdir = np.zeros(n, np.float32)
    cdir[n - 1] = -1.0
    axes = np.eye(n, dtype=np.float32)[: n - 1]
    spec = {
        "n": n,
        "verts": verts,
        "facets": facets,
        "mesh_color": (ALBEDO, ALBEDO, ALBEDO),
        "mesh_diffuse": 1.0,
        "floor": None,
        "light": {"kind": light_kind, "pos": light, "color": (1.0, 1.0, 1.0),
                  "unit": float(np.linalg.norm(light.astype(np.float64)))},
        "projector": {"kind": projector, "org": cam, "dir": cdir, "axes": axes,
                      "param": extent / screen if projector == PARALLEL else 60.0,
                      "screen": [screen] * (n - 1)},
        "bg": {"color": BACKGROUND, "light": True, "light_color": BACKGROUND_LIGHT},
        "spp": spp,
        "max_depth": max_depth,
        "seed": seed,
    }
    if floor:
        org, edges = floor_slab(n)
        spec["floor"] = {"org": org, "edges": edges, "color": (ALBEDO, ALBEDO, ALBEDO), "diffuse": 1.0}
    return spec


def config(name: str, hull: str = "ntrace") -> dict:
    """The measured configurations (full size) and their reduced test-size counterparts.  hull: the
    convex-hull method of the sphere meshes (see sphere_hull; "qhull" keeps the library unloaded)."""
    if name == "n3":
        v, f = icosphere(5)
        return make_spec(3, v, f, screen=400, spp=16)
    if name == "n4":
        v, f = sphere_hull(4, 100_000, seed=0, method=hull)
        return make_spec(4, v, f, screen=128, spp=16)
    if name == "n5":
        v, f = sphere_hull(5, 50_000, seed=0, cap=0.5, method=hull)
        return make_spec(5, v, f, screen=48, spp=4)
    if name == "n6":
        v, f = sphere_hull(6, 400, seed=0, method=hull)
        return make_spec(6, v, f, screen=12, spp=4)
    if name == "n3_small":
        v, f = icosphere(2)
        return make_spec(3, v, f, screen=48, spp=16)
    if name == "n4_small":
        v, f = sphere_hull(4, 800, seed=1, method=hull)
        return make_spec(4, v, f, screen=12, spp=8)
    if name == "n5_small":
        v, f = sphere_hull(5, 300, seed=2, cap=0.5, method=hull)
        return make_spec(5, v, f, screen=6, spp=4)
    if name == "n6_small":
        v, f = sphere_hull(6, 120, seed=3, method=hull)
        return make_spec(6, v, f, screen=4, spp=2)
    raise KeyError(name)


INTERFACE_SCENES = ("constant_light_n4", "perspective_n4", "spherical_n5", "hplt_n4", "two_mesh_n3")


def interface_scene(name: str) -> dict:
    """Small scenes that use the scene types the measured configurations do not: a ConstantLight, the
    perspective and spherical projectors, a hyperplane parallelotope, and two meshes (a closed sphere
    and an open bowl standing on the floor, whose rays start inside the bowl's root box: the sorted
    early break of ray_intersection with the root box's exit distance, ray_intersection.h:26-105)."""
    if name == "constant_light_n4":
        v, f = sphere_hull(4, 800, seed=1)
        spec = make_spec(4, v, f, screen=12, spp=8, light_kind=1)
        spec["light"]["color"] = (0.6, 0.5, 0.4)
        return spec
    if name == "perspective_n4":
        v, f = sphere_hull(4, 800, seed=1)
        spec = make_spec(4, v, f, screen=12, spp=8, projector=PERSPECTIVE)
        spec["projector"]["org"] = np.array([0.3, -0.2, 0.1, 3.5], np.float32)
        spec["projector"]["param"] = 70.0
        return spec
    if name == "spherical_n5":
        v, f = sphere_hull(5, 300, seed=2, cap=0.5)
        spec = make_spec(5, v, f, screen=6, spp=4, projector=SPHERICAL)
        spec["projector"]["org"] = np.array([0.2, 0.1, -0.1, 0.0, 4.0], np.float32)
        spec["projector"]["param"] = 50.0
        return spec
    if name == "hplt_n4":
        v, f = sphere_hull(4, 800, seed=1)
        spec = make_spec(4, v, f, screen=12, spp=8)
        # a slanted three-dimensional wall beside the sphere
        spec["hplt"] = {"org": np.array([1.35, -2.0, -2.0, -1.2], np.float32),
                        "edges": np.array([[0, 4, 0, 0], [0, 0, 4, 0], [0.6, 0, 0, 3.0]], np.float32),
                        "color": (0.8, 0.6, 0.5), "diffuse": 1.0}
        return spec
    if name == "two_mesh_n3":
        bowl_v, bowl_f = sphere_hull(3, 400, seed=7, cap=0.9)  # open at the top
        spec = make_spec(3, bowl_v, bowl_f, screen=24, spp=16, extent=5.0)
        ball_v, ball_f = icosphere(2)
        spec["mesh2"] = {"verts": (ball_v * np.float32(0.6) + np.array([1.5, 1.1, -0.4], np.float32)).astype(np.float32),
                         "facets": ball_f, "color": (0.5, 0.7, 0.6), "diffuse": 1.0}
        return spec
    raise KeyError(name)


def effective_spp(n: int, spp: int) -> int:
    """Samples per pixel after stratification: the smallest k^(n-1) >= spp of the two integers around
    spp^(1/(n-1)) (StratifiedJitteredSampler, src/painter/sampling/sampler.h:31-52); the library's
    nt_effective_spp, restated so that processes that must not load the library can use it."""
    m = n - 1
    v = spp ** (1.0 / m)
    f = math.floor(v)
    return f ** m if f ** m >= spp else math.ceil(v) ** m


def build_scene(spec: dict, threads: int = 0, tree_on_gpu: bool = False, leaf_records: int = 0) -> ntrace.Scene:
    n = spec["n"]
    s = ntrace.Scene(n)
    if spec["verts"] is not None:
        s.add_mesh(spec["verts"], spec["facets"], color=spec["mesh_color"], diffuse=spec["mesh_diffuse"])
        if spec.get("normals") is not None:
            s.set_mesh_normals(0, spec["normals"], spec.get("facet_normals"))
    m2 = spec.get("mesh2")
    if m2 is not None:
        s.add_mesh(m2["verts"], m2["facets"], color=m2["color"], diffuse=m2["diffuse"])
    if spec["floor"] is not None:
        fl = spec["floor"]
        s.add_parallelotope(fl["org"], fl["edges"], color=fl["color"], diffuse=fl["diffuse"])
    hp = spec.get("hplt")
    if hp is not None:
        s.add_hyperplane_parallelotope(hp["org"], hp["edges"], color=hp["color"], diffuse=hp["diffuse"])
    L = spec["light"]
    if L["kind"] == 0:
        s.add_point_light(L["pos"], L["color"], L["unit"])
    else:
        s.add_constant_light(L["pos"], L["color"])
    P = spec["projector"]
    s.set_projector(P["kind"], P["org"], P["dir"], P["axes"], P["param"], P["screen"])
    bg = spec["bg"]
    s.set_background(bg["color"], bg["light"], bg["light_color"])
    s.build(threads, tree_on_gpu=tree_on_gpu, leaf_records=leaf_records)
    return s
