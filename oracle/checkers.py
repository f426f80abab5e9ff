"""ctypes bindings of the two CPU checkers (TEST INFRASTRUCTURE ONLY).

* :class:`Port`      - the C restatement (oracle/ntrace_oracle.c, library oracle/_lib/libntrace_oracle.so)
* :class:`Reference` - the reference painter compiled from its own sources (oracle/ref_bridge.cpp,
                       library oracle/_ref/libref_painter.so)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module; the product
(math_b200) never does.  Scenes are the plain dicts of math_b200.scenes.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "_lib" / "libntrace_oracle.so"
REF_LIB = HERE / "_ref" / "libref_painter.so"
REF_FAST_LIB = HERE / "_ref" / "fast" / "libref_painter.so"


def reference_root() -> Path:
    """The reference checkout: $NTRACE_REFERENCE_ROOT, else the directory "reference" beside this
    checkout (in the same parent directory)."""
    env = os.environ.get("NTRACE_REFERENCE_ROOT")
    return Path(env) if env else HERE.parents[1] / "reference"


def build(ref: bool = True) -> None:
    """Builds the port, and both reference builds (parity: -O2 without contraction; timing: the
    reference's own -Ofast) when the reference sources are present."""
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    root = reference_root()
    if ref and (root / "src" / "painter" / "painter.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "ref_fast", f"REF_ROOT={root}"], check=True)


class SceneStruct(ctypes.Structure):
    """Layout of ort_scene / refb_scene."""

    _fields_ = [
        ("n", ctypes.c_int), ("dbl", ctypes.c_int),
        ("verts", ctypes.c_void_p), ("nverts", ctypes.c_long), ("facets", ctypes.c_void_p), ("nfacets", ctypes.c_long),
        ("mesh_color", ctypes.c_float * 3), ("mesh_diffuse", ctypes.c_float),
        ("has_floor", ctypes.c_int), ("floor_org", ctypes.c_float * 6), ("floor_edges", ctypes.c_float * 36),
        ("floor_color", ctypes.c_float * 3), ("floor_diffuse", ctypes.c_float),
        ("light_kind", ctypes.c_int), ("light_pos", ctypes.c_float * 6), ("light_color", ctypes.c_float * 3),
        ("light_unit_distance", ctypes.c_float),
        ("projector_kind", ctypes.c_int), ("cam_org", ctypes.c_float * 6), ("cam_dir", ctypes.c_float * 6),
        ("screen_axes", ctypes.c_float * 30), ("proj_param", ctypes.c_float), ("screen", ctypes.c_int * 5),
        ("bg_color", ctypes.c_float * 3), ("bg_light_color", ctypes.c_float * 3), ("bg_is_light", ctypes.c_int),
        ("smooth_normal", ctypes.c_int), ("tree_threads", ctypes.c_int),
        ("normals", ctypes.c_void_p), ("nnormals", ctypes.c_long), ("facet_normals", ctypes.c_void_p),
        ("verts2", ctypes.c_void_p), ("nverts2", ctypes.c_long), ("facets2", ctypes.c_void_p), ("nfacets2", ctypes.c_long),
        ("mesh2_color", ctypes.c_float * 3), ("mesh2_diffuse", ctypes.c_float),
        ("has_hplt", ctypes.c_int), ("hplt_org", ctypes.c_float * 6), ("hplt_edges", ctypes.c_float * 30),
        ("hplt_color", ctypes.c_float * 3), ("hplt_diffuse", ctypes.c_float),
    ]


class PortStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_longlong), ("rays", ctypes.c_longlong), ("facet_tests", ctypes.c_longlong),
                ("box_steps", ctypes.c_longlong), ("descent_levels", ctypes.c_longlong),
                ("shadow_rays", ctypes.c_longlong), ("seconds", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class RefStats(ctypes.Structure):
    _fields_ = [("pass_count", ctypes.c_longlong), ("pixel_count", ctypes.c_longlong), ("ray_count", ctypes.c_longlong),
                ("sample_count", ctypes.c_longlong), ("seconds", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def scene_struct(spec: dict, dbl: bool, threads: int = 1) -> tuple[SceneStruct, list]:
    n = spec["n"]
    s = SceneStruct()
    keep = []
    s.n = n
    s.dbl = int(dbl)
    if spec["verts"] is not None:
        v = np.ascontiguousarray(spec["verts"], dtype=np.float32).reshape(-1, n)
        f = np.ascontiguousarray(spec["facets"], dtype=np.int32).reshape(-1, n)
        keep += [v, f]
        s.verts, s.nverts, s.facets, s.nfacets = v.ctypes.data, len(v), f.ctypes.data, len(f)
    for i in range(3):
        s.mesh_color[i] = spec["mesh_color"][i]
    s.mesh_diffuse = spec["mesh_diffuse"]
    if spec["floor"] is not None:
        fl = spec["floor"]
        s.has_floor = 1
        for k in range(n):
            s.floor_org[k] = fl["org"][k]
        e = np.asarray(fl["edges"], np.float32).reshape(n, n)
        for i in range(n):
            for k in range(n):
                s.floor_edges[i * n + k] = e[i, k]
        for i in range(3):
            s.floor_color[i] = fl["color"][i]
        s.floor_diffuse = fl["diffuse"]
    L = spec["light"]
    s.light_kind = L["kind"]
    for k in range(n):
        s.light_pos[k] = L["pos"][k]
    for i in range(3):
        s.light_color[i] = L["color"][i]
    s.light_unit_distance = L["unit"]
    P = spec["projector"]
    s.projector_kind = P["kind"]
    for k in range(n):
        s.cam_org[k] = P["org"][k]
        s.cam_dir[k] = P["dir"][k]
    ax = np.asarray(P["axes"], np.float32).reshape(n - 1, n)
    for j in range(n - 1):
        for k in range(n):
            s.screen_axes[j * n + k] = ax[j, k]
        s.screen[j] = int(P["screen"][j])
    s.proj_param = P["param"]
    bg = spec["bg"]
    for i in range(3):
        s.bg_color[i] = bg["color"][i]
        s.bg_light_color[i] = bg["light_color"][i]
    s.bg_is_light = int(bg["light"])
    s.smooth_normal = int(bool(spec.get("smooth_normal", False)))
    s.tree_threads = threads
    if spec.get("normals") is not None:
        nv = np.ascontiguousarray(spec["normals"], dtype=np.float32).reshape(-1, n)
        keep.append(nv)
        s.normals, s.nnormals = nv.ctypes.data, len(nv)
        if spec.get("facet_normals") is not None:
            fn = np.ascontiguousarray(spec["facet_normals"], dtype=np.int32).reshape(-1, n)
            keep.append(fn)
            s.facet_normals = fn.ctypes.data
    m2 = spec.get("mesh2")
    if m2 is not None:
        v = np.ascontiguousarray(m2["verts"], dtype=np.float32).reshape(-1, n)
        f = np.ascontiguousarray(m2["facets"], dtype=np.int32).reshape(-1, n)
        keep += [v, f]
        s.verts2, s.nverts2, s.facets2, s.nfacets2 = v.ctypes.data, len(v), f.ctypes.data, len(f)
        for i in range(3):
            s.mesh2_color[i] = m2["color"][i]
        s.mesh2_diffuse = m2["diffuse"]
    hp = spec.get("hplt")
    if hp is not None:
        s.has_hplt = 1
        e = np.asarray(hp["edges"], np.float32).reshape(n - 1, n)
        for k in range(n):
            s.hplt_org[k] = hp["org"][k]
        for i in range(n - 1):
            for k in range(n):
                s.hplt_edges[i * n + k] = e[i, k]
        for i in range(3):
            s.hplt_color[i] = hp["color"][i]
        s.hplt_diffuse = hp["diffuse"]
    return s, keep


class _Mesh:
    def __init__(self, owner, handle, n):
        self._owner = owner
        self.h = handle
        self.n = n

    def __del__(self):
        try:
            self._owner._destroy(self.h)
        except Exception:
            pass


class Port:
    """The C restatement: FP64 (dbl=True) mirrors Mesh<N,double>/paint<N,double>, FP32 the float path."""

    def __init__(self):
        if not PORT_LIB.exists():
            build(ref=False)
        lib = ctypes.CDLL(str(PORT_LIB))
        vp = ctypes.c_void_p
        lib.ort_mesh_build.restype = vp
        lib.ort_mesh_build.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_long, vp, ctypes.c_long, ctypes.c_char_p,
                                       ctypes.c_int]
        lib.ort_mesh_destroy.argtypes = [vp]
        lib.ort_mesh_trace.argtypes = [vp, vp, vp, ctypes.c_long, vp, vp, ctypes.POINTER(PortStats)]
        lib.ort_mesh_tree_info.argtypes = [vp, vp, vp, vp]
        lib.ort_mesh_tree_export.argtypes = [vp] * 7
        lib.ort_mesh_facet_export.argtypes = [vp, vp, vp]
        lib.ort_paint.argtypes = [ctypes.POINTER(SceneStruct), ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, vp,
                                  ctypes.c_long, ctypes.c_longlong, vp, ctypes.POINTER(PortStats), ctypes.c_char_p,
                                  ctypes.c_int]
        lib.ort_effective_spp.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.ort_philox.argtypes = [ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        lib.ort_cosine_sphere_coefficient.argtypes = [ctypes.c_int]
        lib.ort_cosine_sphere_coefficient.restype = ctypes.c_double
        lib.ort_cosine_hemisphere.argtypes = [ctypes.c_int, vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, vp]
        self.lib = lib

    def _destroy(self, h):
        self.lib.ort_mesh_destroy(h)

    def mesh(self, n: int, verts, facets, dbl: bool = True) -> _Mesh:
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, n)
        f = np.ascontiguousarray(facets, np.int32).reshape(-1, n)
        err = ctypes.create_string_buffer(512)
        h = self.lib.ort_mesh_build(n, int(dbl), v.ctypes.data, len(v), f.ctypes.data, len(f), err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        return _Mesh(self, h, n)

    def trace(self, mesh: _Mesh, org, dirs):
        o = np.ascontiguousarray(org, np.float32).reshape(-1, mesh.n)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, mesh.n)
        fo = np.zeros(len(o), np.int32)
        to = np.zeros(len(o), np.float64)
        st = PortStats()
        self.lib.ort_mesh_trace(mesh.h, o.ctypes.data, d.ctypes.data, len(o), fo.ctypes.data, to.ctypes.data,
                                ctypes.byref(st))
        return fo, to, st.as_dict()

    def tree(self, mesh: _Mesh) -> dict:
        bc, ic, dist = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        self.lib.ort_mesh_tree_info(mesh.h, ctypes.byref(bc), ctypes.byref(ic), ctypes.byref(dist))
        n = mesh.n
        org = np.zeros((bc.value, n))
        size = np.zeros((bc.value, n))
        first = np.zeros(bc.value, np.int32)
        depth = np.zeros(bc.value, np.int32)
        off = np.zeros(bc.value + 1, np.int64)
        idx = np.zeros(max(1, ic.value), np.int32)
        self.lib.ort_mesh_tree_export(mesh.h, org.ctypes.data, size.ctypes.data, first.ctypes.data, depth.ctypes.data,
                                      off.ctypes.data, idx.ctypes.data)
        return {"org": org, "size": size, "first_child": first, "depth": depth, "offset": off,
                "indices": idx[: ic.value], "distance_from_facet": dist.value}

    def paint(self, spec: dict, dbl: bool, spp: int | None = None, max_depth: int | None = None, seed: int | None = None,
              threads: int = 1, pixels=None, sample_offset: int = 0):
        s, keep = scene_struct(spec, dbl)
        spp = spec["spp"] if spp is None else spp
        max_depth = spec["max_depth"] if max_depth is None else max_depth
        seed = spec["seed"] if seed is None else seed
        n = spec["n"]
        total = int(np.prod(spec["projector"]["screen"]))
        if pixels is not None:
            px = np.ascontiguousarray(pixels, np.int32).reshape(-1, n - 1)
            npix = len(px)
            pptr = px.ctypes.data
        else:
            px, npix, pptr = None, total, None
        out = np.zeros((npix, 3), np.float32)
        st = PortStats()
        err = ctypes.create_string_buffer(512)
        rc = self.lib.ort_paint(ctypes.byref(s), spp, max_depth, seed & (2 ** 64 - 1), threads, pptr, npix, sample_offset,
                                out.ctypes.data, ctypes.byref(st), err, 512)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out, st.as_dict()

    def philox(self, key: int, ctr) -> np.ndarray:
        c = np.ascontiguousarray(ctr, np.uint32)
        out = np.zeros(4, np.uint32)
        self.lib.ort_philox(key & 0xFFFFFFFF, (key >> 32) & 0xFFFFFFFF, c.ctypes.data, out.ctypes.data)
        return out

    def effective_spp(self, n: int, spp: int) -> int:
        return self.lib.ort_effective_spp(n, spp)

    def cosine_sphere_coefficient(self, n: int) -> float:
        return self.lib.ort_cosine_sphere_coefficient(n)

    def cosine_hemisphere(self, n: int, normal, seed: int, path: int, stream: int) -> np.ndarray | None:
        nrm = np.ascontiguousarray(normal, np.float64)
        out = np.zeros(n, np.float64)
        ok = self.lib.ort_cosine_hemisphere(n, nrm.ctypes.data, seed, path, stream, out.ctypes.data)
        return out if ok else None


class Reference:
    """The reference painter compiled from its own sources (available where it was built)."""

    @staticmethod
    def available(fast: bool = False) -> bool:
        return (REF_FAST_LIB if fast else REF_LIB).exists()

    def __init__(self, fast: bool = False):
        """fast=False: the parity build (IEEE order); fast=True: the reference's own -Ofast -mavx -mfma
        build, for timing."""
        path = REF_FAST_LIB if fast else REF_LIB
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (the reference sources are needed to build it)")
        self.path = path
        self.flags = "-Ofast -mavx -mfma" if fast else "-O2 -mavx -mfma -ffp-contract=off"
        lib = ctypes.CDLL(str(path))
        vp = ctypes.c_void_p
        lib.refb_mesh_create.restype = vp
        lib.refb_mesh_create.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_long, vp, ctypes.c_long, ctypes.c_int,
                                         ctypes.c_char_p, ctypes.c_int]
        lib.refb_mesh_destroy.argtypes = [vp]
        lib.refb_mesh_trace.argtypes = [vp, vp, vp, ctypes.c_long, vp, vp]
        lib.refb_mesh_tree_info.argtypes = [vp, vp, vp, vp]
        lib.refb_mesh_tree_export.argtypes = [vp] * 6
        lib.refb_paint.argtypes = [ctypes.POINTER(SceneStruct), ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_int,
                                   vp, ctypes.c_long, ctypes.c_int, vp, ctypes.POINTER(RefStats), ctypes.c_char_p,
                                   ctypes.c_int]
        self.lib = lib

    def _destroy(self, h):
        self.lib.refb_mesh_destroy(h)

    def mesh(self, n: int, verts, facets, dbl: bool = True, threads: int = 0) -> _Mesh:
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, n)
        f = np.ascontiguousarray(facets, np.int32).reshape(-1, n)
        err = ctypes.create_string_buffer(512)
        h = self.lib.refb_mesh_create(n, int(dbl), v.ctypes.data, len(v), f.ctypes.data, len(f),
                                      threads or os.cpu_count() or 1, err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        return _Mesh(self, h, n)

    def trace(self, mesh: _Mesh, org, dirs):
        o = np.ascontiguousarray(org, np.float32).reshape(-1, mesh.n)
        d = np.ascontiguousarray(dirs, np.float32).reshape(-1, mesh.n)
        fo = np.zeros(len(o), np.int32)
        to = np.zeros(len(o), np.float64)
        self.lib.refb_mesh_trace(mesh.h, o.ctypes.data, d.ctypes.data, len(o), fo.ctypes.data, to.ctypes.data)
        return fo, to

    def tree_info(self, mesh: _Mesh) -> dict:
        bc, ic, dist = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
        self.lib.refb_mesh_tree_info(mesh.h, ctypes.byref(bc), ctypes.byref(ic), ctypes.byref(dist))
        return {"box_count": bc.value, "index_count": ic.value, "distance_from_facet": dist.value}

    def paint(self, spec: dict, dbl: bool, spp: int | None = None, max_depth: int | None = None, seed: int = 1,
              threads: int = 1, pixels=None, bar_height: int = 20, store: bool = True):
        s, keep = scene_struct(spec, dbl, threads=os.cpu_count() or 1)
        spp = spec["spp"] if spp is None else spp
        max_depth = spec["max_depth"] if max_depth is None else max_depth
        n = spec["n"]
        total = int(np.prod(spec["projector"]["screen"]))
        if pixels is not None:
            px = np.ascontiguousarray(pixels, np.int32).reshape(-1, n - 1)
            npix, pptr = len(px), px.ctypes.data
        else:
            px, npix, pptr = None, total, None
        out = np.zeros((npix, 3), np.float32) if store else None
        st = RefStats()
        err = ctypes.create_string_buffer(1024)
        rc = self.lib.refb_paint(ctypes.byref(s), spp, max_depth, seed, threads, pptr, npix, bar_height,
                                 out.ctypes.data if store else None, ctypes.byref(st), err, 1024)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out, st.as_dict()
