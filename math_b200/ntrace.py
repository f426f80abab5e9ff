"""Python mirror of the painter interface over the C ABI (include/ntrace.h).

The reference assembles a PaintObjects<N,T> from visible shapes, light sources, a projector and the
default surface (src/painter/objects.h:141-223) and calls paint<N,T>() (src/painter/painter.cpp:599-625).
:class:`Scene` keeps that vocabulary: ``add_mesh`` (VisibleSharedMesh over Mesh<N,T>),
``add_parallelotope`` (VisibleParallelotope), ``add_hyperplane_parallelotope``
(VisibleHyperplaneParallelotope), ``add_point_light`` / ``add_constant_light``, ``set_projector``
(Visible{Parallel,Perspective,Spherical}Projector), ``set_background`` (default surface properties),
then ``build`` and ``render``.  Errors raise :class:`NtraceError`, carrying the library's message, as
paint() reports through its notifier.

The library is the in-tree ``libntrace.so``; there is no fallback implementation: if it cannot be
loaded, every call raises.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libntrace.so"

NT_OK, NT_EINVAL, NT_EDEGENERATE, NT_ECUDA, NT_ETIMEOUT, NT_ESTOPPED, NT_ENOMEM, NT_ESTATE = range(8)
PARALLEL, PERSPECTIVE, SPHERICAL = 0, 1, 2

EXPORTED_SYMBOLS = (
    "nt_scene_create", "nt_scene_destroy", "nt_scene_add_mesh", "nt_scene_add_parallelotope",
    "nt_scene_add_hyperplane_parallelotope", "nt_scene_add_point_light", "nt_scene_add_constant_light",
    "nt_scene_set_projector", "nt_scene_set_background", "nt_scene_build", "nt_scene_mesh_info", "nt_render",
    "nt_accum_clear", "nt_accum_read", "nt_scene_pixel_count", "nt_trace_closest", "nt_trace_closest_device",
    "nt_scene_tree_export", "nt_last_error_message", "nt_effective_spp", "nt_cosine_sphere_coefficient",
    "nt_scene_upload", "nt_scene_upload_begin", "nt_scene_upload_commit", "nt_scene_stream", "nt_scene_set_mesh_normals", "nt_scene_add_obj_file", "nt_scene_dimension",
    "nt_scene_object_count", "nt_accum_read_srgb_slice", "nt_convex_hull", "nt_hull_facet_count", "nt_hull_facets",
    "nt_hull_destroy", "nt_scene_clear_lights", "nt_render_batch",
    "nt_autotune", "nt_scene_set_object_surface", "nt_render_aux",
    "nt_render_moments", "nt_render_noalloc", "nt_render_pixels", "nt_probe_peaks",
    "nt_denoiser_create", "nt_denoiser_destroy", "nt_denoiser_get_layout", "nt_denoiser_get_params",
    "nt_denoiser_set_params", "nt_denoiser_set_input", "nt_denoiser_apply", "nt_denoiser_gradient",
    "nt_denoiser_train_step", "nt_tc_gemm_bf16", "nt_tc_gemm_bf16_t", "nt_tc_gemm_wait_selftest",
)


class NtraceError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"ntrace error {code}: {message}")
        self.code = code


class Surface(ctypes.Structure):
    _fields_ = [("color", ctypes.c_float * 3), ("diffuse", ctypes.c_float), ("light_source", ctypes.c_int),
                ("light_color", ctypes.c_float * 3)]


class BuildOpts(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("host_only", ctypes.c_int), ("tree_on_gpu", ctypes.c_int),
                ("leaf_records", ctypes.c_int)]


class RenderOpts(ctypes.Structure):
    _fields_ = [("samples_per_pixel", ctypes.c_int), ("max_depth", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("retest", ctypes.c_int), ("smooth_normal", ctypes.c_int), ("pool_paths", ctypes.c_int64),
                ("timing", ctypes.c_int), ("stop", ctypes.c_void_p), ("graph_iterations", ctypes.c_int),
                ("sample_offset", ctypes.c_int64), ("walk_chunk", ctypes.c_int), ("walk_small_leaf", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_int64), ("rays", ctypes.c_int64), ("shadow_rays", ctypes.c_int64),
                ("facet_tests", ctypes.c_int64), ("box_steps", ctypes.c_int64), ("retests", ctypes.c_int64),
                ("descent_levels", ctypes.c_int64), ("error_bits", ctypes.c_int64), ("spp_effective", ctypes.c_int),
                ("seconds", ctypes.c_double), ("raygen_ms", ctypes.c_double), ("extend_ms", ctypes.c_double),
                ("shade_ms", ctypes.c_double), ("shadow_ms", ctypes.c_double), ("launches", ctypes.c_int64),
                ("extend_launches", ctypes.c_int64), ("shadow_launches", ctypes.c_int64),
                ("shadow_facet_tests", ctypes.c_int64), ("shadow_box_steps", ctypes.c_int64),
                ("shadow_retests", ctypes.c_int64), ("shadow_descent_levels", ctypes.c_int64),
                ("iterations", ctypes.c_int64), ("plan_ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Peaks(ctypes.Structure):
    _fields_ = [("l2_read_gbs", ctypes.c_double), ("fp32_fma_tflops", ctypes.c_double), ("l2_ms", ctypes.c_double),
                ("fma_ms", ctypes.c_double)]


def probe_peaks() -> dict:
    """L2 read bandwidth (GB/s) and FP32 FMA rate (TFLOP/s) of the current GPU (nt_probe_peaks)."""
    p = Peaks()
    _check(library().nt_probe_peaks(ctypes.byref(p)))
    return {name: getattr(p, name) for name, _ in Peaks._fields_}


class MeshInfo(ctypes.Structure):
    _fields_ = [("facet_count", ctypes.c_int64), ("node_count", ctypes.c_int64), ("leaf_count", ctypes.c_int64),
                ("index_count", ctypes.c_int64), ("max_depth", ctypes.c_int), ("distance_from_facet", ctypes.c_double),
                ("degenerate_facets", ctypes.c_int64), ("build_seconds", ctypes.c_double),
                ("device_bytes", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def library() -> ctypes.CDLL:
    """Loads libntrace.so (building it first if the sources are newer and nvcc is present)."""
    global _lib
    if _lib is not None:
        return _lib
    if os.environ.get("NTRACE_NO_BUILD") != "1":
        try:
            from . import build as _build
            _build.build()
        except Exception:
            if not LIB_PATH.exists():
                raise
    if not LIB_PATH.exists():
        raise NtraceError(NT_ESTATE, f"{LIB_PATH} is missing; run math_b200/build.py")
    lib = ctypes.CDLL(str(LIB_PATH))
    vp, i64, f32p, i32p = ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p
    sig = {
        "nt_scene_create": ([ctypes.c_int, ctypes.POINTER(vp)], ctypes.c_int),
        "nt_scene_destroy": ([vp], ctypes.c_int),
        "nt_scene_add_mesh": ([vp, f32p, i64, i32p, i64, ctypes.POINTER(Surface)], ctypes.c_int),
        "nt_scene_add_parallelotope": ([vp, f32p, f32p, ctypes.POINTER(Surface)], ctypes.c_int),
        "nt_scene_add_hyperplane_parallelotope": ([vp, f32p, f32p, ctypes.POINTER(Surface)], ctypes.c_int),
        "nt_scene_add_point_light": ([vp, f32p, f32p, ctypes.c_float], ctypes.c_int),
        "nt_scene_add_constant_light": ([vp, f32p, f32p], ctypes.c_int),
        "nt_scene_set_projector": ([vp, ctypes.c_int, f32p, f32p, f32p, ctypes.c_float, i32p], ctypes.c_int),
        "nt_scene_set_background": ([vp, ctypes.POINTER(Surface)], ctypes.c_int),
        "nt_scene_build": ([vp, ctypes.POINTER(BuildOpts)], ctypes.c_int),
        "nt_scene_mesh_info": ([vp, ctypes.c_int, ctypes.POINTER(MeshInfo)], ctypes.c_int),
        "nt_render": ([vp, ctypes.POINTER(RenderOpts), ctypes.POINTER(Stats)], ctypes.c_int),
        "nt_accum_clear": ([vp], ctypes.c_int),
        "nt_accum_read": ([vp, f32p, ctypes.POINTER(i64)], ctypes.c_int),
        "nt_scene_pixel_count": ([vp], i64),
        "nt_scene_upload": ([vp, ctypes.POINTER(i64)], ctypes.c_int),
        "nt_scene_upload_begin": ([vp, ctypes.POINTER(i64)], ctypes.c_int),
        "nt_scene_upload_commit": ([vp], ctypes.c_int),
        "nt_scene_stream": ([vp], vp),
        "nt_trace_closest": ([vp, ctypes.c_int, f32p, f32p, i64, ctypes.c_int, i32p, f32p, ctypes.POINTER(Stats)],
                             ctypes.c_int),
        "nt_trace_closest_device": ([vp, ctypes.c_int, vp, vp, i64, ctypes.c_int, vp, vp, vp], ctypes.c_int),
        "nt_scene_tree_export": ([vp, ctypes.c_int, i32p, i32p, f32p, f32p], ctypes.c_int),
        "nt_last_error_message": ([], ctypes.c_char_p),
        "nt_effective_spp": ([ctypes.c_int, ctypes.c_int], ctypes.c_int),
        "nt_cosine_sphere_coefficient": ([ctypes.c_int], ctypes.c_double),
        "nt_scene_set_mesh_normals": ([vp, ctypes.c_int, f32p, i64, i32p], ctypes.c_int),
        "nt_scene_add_obj_file": ([vp, ctypes.c_char_p, ctypes.POINTER(Surface)], ctypes.c_int),
        "nt_scene_dimension": ([vp], ctypes.c_int),
        "nt_accum_read_srgb_slice": ([vp, i32p, vp, ctypes.c_int], ctypes.c_int),
        "nt_convex_hull": ([ctypes.c_int, f32p, i64, ctypes.POINTER(vp)], ctypes.c_int),
        "nt_hull_facet_count": ([vp], i64),
        "nt_hull_facets": ([vp, i32p], ctypes.c_int),
        "nt_hull_destroy": ([vp], ctypes.c_int),
        "nt_scene_object_count": ([vp], ctypes.c_int),
        "nt_scene_clear_lights": ([vp], ctypes.c_int),
        "nt_render_batch": ([ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(RenderOpts), ctypes.POINTER(Stats)],
                            ctypes.c_int),
        "nt_autotune": ([vp, ctypes.POINTER(RenderOpts), ctypes.POINTER(RenderOpts), ctypes.POINTER(ctypes.c_double)],
                        ctypes.c_int),
        "nt_scene_set_object_surface": ([vp, ctypes.c_int, ctypes.POINTER(Surface)], ctypes.c_int),
        "nt_render_aux": ([vp, vp, vp, vp], ctypes.c_int),
        "nt_render_moments": ([vp, ctypes.POINTER(RenderOpts), i64, vp, vp, ctypes.POINTER(Stats)], ctypes.c_int),
        "nt_render_pixels": ([vp, ctypes.POINTER(RenderOpts), vp, i64, vp, ctypes.POINTER(Stats)], ctypes.c_int),
        "nt_probe_peaks": ([ctypes.POINTER(Peaks)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(code: int) -> None:
    if code != NT_OK:
        msg = library().nt_last_error_message()
        raise NtraceError(code, msg.decode() if msg else "")


def _f32(a, shape=None) -> np.ndarray:
    arr = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if shape is not None:
        arr = arr.reshape(shape)
    return arr


def _surface(color=(1.0, 1.0, 1.0), diffuse=1.0, light_source=False, light_color=(0.0, 0.0, 0.0)) -> Surface:
    s = Surface()
    for i in range(3):
        s.color[i] = float(color[i])
        s.light_color[i] = float(light_color[i])
    s.diffuse = float(diffuse)
    s.light_source = int(bool(light_source))
    return s


def convex_hull(points) -> np.ndarray:
    """Boundary facets (point indices, facet_count x n) of the convex hull of points (count x n)."""
    lib = library()
    p = _f32(points)
    n = p.shape[1]
    h = ctypes.c_void_p()
    _check(lib.nt_convex_hull(n, p.ctypes.data, len(p), ctypes.byref(h)))
    try:
        out = np.zeros((lib.nt_hull_facet_count(h), n), np.int32)
        _check(lib.nt_hull_facets(h, out.ctypes.data))
    finally:
        lib.nt_hull_destroy(h)
    return out


def effective_spp(n: int, spp: int) -> int:
    return library().nt_effective_spp(n, spp)


def cosine_sphere_coefficient(n: int) -> float:
    return library().nt_cosine_sphere_coefficient(n)


def render_opts(samples_per_pixel: int, max_depth: int = 100, seed: int = 0, retest: bool = True,
                smooth_normal: bool = False, pool_paths: int = 0, timing: bool = False,
                graph_iterations: int = 0, sample_offset: int = 0, walk_chunk: int = 0,
                walk_small_leaf: int = 0) -> RenderOpts:
    return RenderOpts(int(samples_per_pixel), int(max_depth), int(seed) & (2 ** 64 - 1), int(bool(retest)),
                      int(bool(smooth_normal)), int(pool_paths), int(bool(timing)), None, int(graph_iterations),
                      int(sample_offset), int(walk_chunk), int(walk_small_leaf))


def render_batch(scenes: list, opts: list[dict]) -> list[dict]:
    """One pass of each scene, run side by side in one CUDA graph (nt_render_batch); opts[i] holds
    the keyword arguments of Scene.render for scene i."""
    lib = library()
    n = len(scenes)
    handles = (ctypes.c_void_p * n)(*[sc._h.value for sc in scenes])
    arr = (RenderOpts * n)(*[render_opts(**o) for o in opts])
    st = (Stats * n)()
    _check(lib.nt_render_batch(handles, n, arr, st))
    return [st[i].as_dict() for i in range(n)]


class Scene:
    """One PaintObjects: objects, light sources, projector and background, in n dimensions."""

    def __init__(self, n: int):
        self.n = int(n)
        self._lib = library()
        h = ctypes.c_void_p()
        _check(self._lib.nt_scene_create(self.n, ctypes.byref(h)))
        self._h = h
        self.screen: tuple[int, ...] = ()
        self._keep: list = []

    def close(self) -> None:
        if self._h:
            self._lib.nt_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- assembly ----
    def add_mesh(self, vertices, facets, color=(1.0, 1.0, 1.0), diffuse=1.0, light_source=False,
                 light_color=(0.0, 0.0, 0.0)) -> None:
        v = _f32(vertices).reshape(-1, self.n)
        f = np.ascontiguousarray(np.asarray(facets, dtype=np.int32)).reshape(-1, self.n)
        s = _surface(color, diffuse, light_source, light_color)
        _check(self._lib.nt_scene_add_mesh(self._h, v.ctypes.data, len(v), f.ctypes.data, len(f), ctypes.byref(s)))

    def add_parallelotope(self, org, edges, color=(1.0, 1.0, 1.0), diffuse=1.0, light_source=False,
                          light_color=(0.0, 0.0, 0.0)) -> None:
        o = _f32(org, (self.n,))
        e = _f32(edges, (self.n, self.n))
        s = _surface(color, diffuse, light_source, light_color)
        _check(self._lib.nt_scene_add_parallelotope(self._h, o.ctypes.data, e.ctypes.data, ctypes.byref(s)))

    def add_hyperplane_parallelotope(self, org, edges, color=(1.0, 1.0, 1.0), diffuse=1.0, light_source=False,
                                     light_color=(0.0, 0.0, 0.0)) -> None:
        o = _f32(org, (self.n,))
        e = _f32(edges, (self.n - 1, self.n))
        s = _surface(color, diffuse, light_source, light_color)
        _check(self._lib.nt_scene_add_hyperplane_parallelotope(self._h, o.ctypes.data, e.ctypes.data, ctypes.byref(s)))

    def add_point_light(self, location, rgb, unit_intensity_distance: float) -> None:
        loc = _f32(location, (self.n,))
        c = _f32(rgb, (3,))
        _check(self._lib.nt_scene_add_point_light(self._h, loc.ctypes.data, c.ctypes.data,
                                                  float(unit_intensity_distance)))

    def add_constant_light(self, location, rgb) -> None:
        loc = _f32(location, (self.n,))
        c = _f32(rgb, (3,))
        _check(self._lib.nt_scene_add_constant_light(self._h, loc.ctypes.data, c.ctypes.data))

    def set_projector(self, kind: int, camera_org, camera_dir, screen_axes, param: float, screen_size) -> None:
        o = _f32(camera_org, (self.n,))
        d = _f32(camera_dir, (self.n,))
        a = _f32(screen_axes, (self.n - 1, self.n))
        sz = np.ascontiguousarray(np.asarray(screen_size, dtype=np.int32).reshape(self.n - 1))
        _check(self._lib.nt_scene_set_projector(self._h, int(kind), o.ctypes.data, d.ctypes.data, a.ctypes.data,
                                                float(param), sz.ctypes.data))
        self.screen = tuple(int(x) for x in sz)

    def set_background(self, color, light_source=False, light_color=(0.0, 0.0, 0.0)) -> None:
        s = _surface(color, 1.0, light_source, light_color)
        _check(self._lib.nt_scene_set_background(self._h, ctypes.byref(s)))

    def build(self, threads: int = 0, host_only: bool = False, tree_on_gpu: bool = False,
              leaf_records: int = 0) -> None:
        """Facet setup and 2^n-trees (on the GPU with tree_on_gpu), then the upload.  leaf_records: 0 keeps
        the leaf-ordered copy of the facet records when it fits a quarter of the free device memory,
        -1 never (nt_build_opts.leaf_records)."""
        o = BuildOpts(threads, int(bool(host_only)), int(bool(tree_on_gpu)), int(leaf_records))
        _check(self._lib.nt_scene_build(self._h, ctypes.byref(o)))

    # ---- queries ----
    def mesh_info(self, mesh_index: int = 0) -> dict:
        info = MeshInfo()
        _check(self._lib.nt_scene_mesh_info(self._h, mesh_index, ctypes.byref(info)))
        return info.as_dict()

    def tree_export(self, mesh_index: int = 0) -> dict:
        info = self.mesh_info(mesh_index)
        nodes = np.zeros((info["node_count"], 2), np.int32)
        idx = np.zeros(max(1, info["index_count"]), np.int32)
        sizes = np.zeros((info["max_depth"] + 1, self.n), np.float32)
        root = np.zeros(self.n, np.float32)
        _check(self._lib.nt_scene_tree_export(self._h, mesh_index, nodes.ctypes.data, idx.ctypes.data,
                                              sizes.ctypes.data, root.ctypes.data))
        return {"nodes": nodes, "indices": idx[: info["index_count"]], "level_sizes": sizes, "root_org": root,
                "distance_from_facet": info["distance_from_facet"]}

    @property
    def pixel_count(self) -> int:
        return int(self._lib.nt_scene_pixel_count(self._h))

    @property
    def stream(self) -> int:
        """The scene's CUDA stream handle (as an integer)."""
        return int(self._lib.nt_scene_stream(self._h) or 0)

    def upload(self) -> int:
        """Re-copies the scene's device arrays from the pinned host copy; returns the bytes moved."""
        b = ctypes.c_int64()
        _check(self._lib.nt_scene_upload(self._h, ctypes.byref(b)))
        return int(b.value)

    def upload_begin(self) -> int:
        """Queues the copy of the scene's arrays into the device staging buffers on the scene's copy
        stream (overlapping a render in flight); returns the bytes queued."""
        b = ctypes.c_int64()
        _check(self._lib.nt_scene_upload_begin(self._h, ctypes.byref(b)))
        return int(b.value)

    def upload_commit(self) -> None:
        """Moves the staged arrays into the live ones, ordered before the next render."""
        _check(self._lib.nt_scene_upload_commit(self._h))

    def render(self, samples_per_pixel: int, max_depth: int = 100, seed: int = 0, retest: bool = True,
               smooth_normal: bool = False, pool_paths: int = 0, timing: bool = False, stop=None,
               graph_iterations: int = 0, sample_offset: int = 0, walk_chunk: int = 0,
               walk_small_leaf: int = 0) -> dict:
        """One pass added to the accumulator (nt_render); sample_offset > 0 starts it at that sample
        index, 0 continues after the accumulated samples."""
        o = render_opts(samples_per_pixel, max_depth, seed, retest, smooth_normal, pool_paths, timing,
                        graph_iterations, sample_offset, walk_chunk, walk_small_leaf)
        if stop is not None:
            o.stop = ctypes.cast(stop, ctypes.c_void_p)
        st = Stats()
        _check(self._lib.nt_render(self._h, ctypes.byref(o), ctypes.byref(st)))
        return st.as_dict()

    def render_pixels(self, pixels, samples_per_pixel: int, max_depth: int = 100, seed: int = 0,
                      retest: bool = True, smooth_normal: bool = False, pool_paths: int = 0,
                      sample_offset: int = 0) -> tuple[np.ndarray, dict]:
        """Mean colour of each listed pixel over samples [sample_offset, + effective spp)
        (nt_render_pixels).  pixels: linear indices, or an (m, n-1) array of screen coordinates."""
        px = np.asarray(pixels)
        if px.ndim == 2:
            strides = np.cumprod([1] + list(self.screen[:-1]), dtype=np.int64)
            px = (px.astype(np.int64) * strides).sum(axis=1)
        lin = np.ascontiguousarray(px, dtype=np.int64).reshape(-1)
        out = np.zeros((len(lin), 3), np.float32)
        o = render_opts(samples_per_pixel, max_depth, seed, retest, smooth_normal, pool_paths, False, 0,
                        sample_offset)
        st = Stats()
        _check(self._lib.nt_render_pixels(self._h, ctypes.byref(o), lin.ctypes.data, len(lin), out.ctypes.data,
                                          ctypes.byref(st)))
        return out, st.as_dict()

    def autotune(self, samples_per_pixel: int, max_depth: int = 100, seed: int = 0, retest: bool = True,
                 smooth_normal: bool = False) -> tuple[dict, float]:
        """Fastest pool size, iterations per graph launch and walk staging chunk for passes of
        samples_per_pixel (probe passes; clears the accumulator).  Returns ({pool_paths,
        graph_iterations, walk_chunk}, pass ms)."""
        base = render_opts(samples_per_pixel, max_depth, seed, retest, smooth_normal, 0, False, 0)
        out = RenderOpts()
        ms = ctypes.c_double()
        _check(self._lib.nt_autotune(self._h, ctypes.byref(base), ctypes.byref(out), ctypes.byref(ms)))
        return {"pool_paths": int(out.pool_paths), "graph_iterations": int(out.graph_iterations),
                "walk_chunk": int(out.walk_chunk), "walk_small_leaf": int(out.walk_small_leaf)}, float(ms.value)

    def clear(self) -> None:
        _check(self._lib.nt_accum_clear(self._h))

    def image(self, out=None) -> tuple[np.ndarray, int]:
        """Mean colour per pixel, shape (pixels, 3), x0 fastest; and samples per pixel.  out: an
        optional float32 array of that shape to fill (e.g. a pinned buffer reused every frame)."""
        if out is None:
            out = np.zeros((self.pixel_count, 3), np.float32)
        elif out.dtype != np.float32 or out.shape != (self.pixel_count, 3) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 array of shape (pixels, 3)")
        spp = ctypes.c_int64()
        _check(self._lib.nt_accum_read(self._h, out.ctypes.data, ctypes.byref(spp)))
        return out, int(spp.value)

    def add_obj_file(self, path, color=(1.0, 1.0, 1.0), diffuse=1.0, light_source=False,
                     light_color=(0.0, 0.0, 0.0)) -> int:
        """Mesh from an OBJ / OBJ-n file; returns its object index."""
        s = _surface(color, diffuse, light_source, light_color)
        _check(self._lib.nt_scene_add_obj_file(self._h, str(path).encode(), ctypes.byref(s)))
        return self._lib.nt_scene_object_count(self._h) - 1

    def set_mesh_normals(self, obj: int, normals, facet_normals=None) -> None:
        """Vertex normals of mesh object `obj` (normal_count x n) and optional per-facet normal indices
        (facet_count x n; default: the facets' vertex indices); used with smooth_normal."""
        nv = _f32(normals).reshape(-1, self.n)
        fn = None if facet_normals is None else np.ascontiguousarray(np.asarray(facet_normals, np.int32))
        _check(self._lib.nt_scene_set_mesh_normals(self._h, int(obj), nv.ctypes.data, len(nv),
                                                   None if fn is None else fn.ctypes.data))

    def clear_lights(self) -> None:
        """Removes every light (add new ones, then build again; the meshes' trees are kept)."""
        _check(self._lib.nt_scene_clear_lights(self._h))

    def set_object_surface(self, obj: int, color=(1.0, 1.0, 1.0), diffuse=1.0, light_source=False,
                           light_color=(0.0, 0.0, 0.0)) -> None:
        s = _surface(color, diffuse, light_source, light_color)
        _check(self._lib.nt_scene_set_object_surface(self._h, int(obj), ctypes.byref(s)))

    def render_aux(self, d_normal: int, d_depth: int, stream: int = 0) -> None:
        """First-hit normal (pixels x n) and depth (pixels) into device arrays (pointers as integers)."""
        _check(self._lib.nt_render_aux(self._h, d_normal, d_depth, stream or None))

    def render_moments(self, samples_per_pixel: int, d_mean: int, d_var: int, sample_offset: int = 0,
                       max_depth: int = 100, seed: int = 0, retest: bool = True) -> dict:
        """One pass of samples_per_pixel: per-pixel mean and variance of the mean into device arrays."""
        o = RenderOpts(int(samples_per_pixel), int(max_depth), int(seed) & (2 ** 64 - 1), int(bool(retest)), 0, 0, 0,
                       None)
        st = Stats()
        _check(self._lib.nt_render_moments(self._h, ctypes.byref(o), int(sample_offset), d_mean, d_var, ctypes.byref(st)))
        return st.as_dict()

    def srgb_slice(self, slice_pos=()) -> np.ndarray:
        """The painter window's view of a 2-D slice: (height, width) words 0x00RRGGBB, row 0 the
        screen's last row; slice_pos fixes screen axes 2.. (n - 3 values)."""
        sl = np.ascontiguousarray(np.asarray(slice_pos, np.int32))
        width, height = self.screen[0], self.screen[1]
        out = np.zeros((height, width), np.uint32)
        _check(self._lib.nt_accum_read_srgb_slice(self._h, sl.ctypes.data if sl.size else None, out.ctypes.data, 0))
        return out

    def trace_closest(self, org, dirs, mesh_index: int = 0, retest: bool = True):
        """Closest facet per ray (-1 = miss) and distance; plus the call's statistics."""
        o = _f32(org).reshape(-1, self.n)
        d = _f32(dirs).reshape(-1, self.n)
        if o.shape != d.shape:
            raise ValueError("org and dirs differ in shape")
        facet = np.zeros(len(o), np.int32)
        t = np.zeros(len(o), np.float32)
        st = Stats()
        _check(self._lib.nt_trace_closest(self._h, mesh_index, o.ctypes.data, d.ctypes.data, len(o), int(bool(retest)),
                                          facet.ctypes.data, t.ctypes.data, ctypes.byref(st)))
        return facet, t, st.as_dict()

    def trace_closest_device(self, d_org: int, d_dir: int, count: int, d_facet: int, d_t: int, mesh_index: int = 0,
                             retest: bool = True, stream: int = 0) -> None:
        """Device-pointer variant (pointers as integers, e.g. torch tensor data_ptr())."""
        _check(self._lib.nt_trace_closest_device(self._h, mesh_index, d_org, d_dir, count, int(bool(retest)), d_facet,
                                                 d_t, stream or None))
