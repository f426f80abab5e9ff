"""OBJ / OBJ-n mesh files (nt_scene_add_obj_file): the geometry the reference's loader reads
(src/obj/file/file_load.cpp): vertices, vertex normals, facets with fan splitting of polygons,
1-based and negative indices; the mesh and tree are the same as from arrays."""

import numpy as np
import pytest


def _write_obj(path, verts, facets, normals=None, negative=False):
    n = verts.shape[1]
    lines = ["# test mesh", "o thing"]
    lines += ["v " + " ".join(f"{x:.9g}" for x in v) for v in verts]
    if normals is not None:
        lines += ["vn " + " ".join(f"{x:.9g}" for x in v) for v in normals]
    lines.append("vt 0.5 0.5")
    nv = len(verts)
    for f in facets:
        idx = [(i - nv) if negative else (i + 1) for i in f]
        if normals is not None:
            lines.append("f " + " ".join(f"{i}/1/{i}" for i in idx))
        else:
            lines.append("f " + " ".join(str(i) for i in idx))
    path.write_text("\n".join(lines) + "\n")


def _scene_from(n, build):
    from math_b200 import ntrace

    s = ntrace.Scene(n)
    build(s)
    s.add_point_light([2.0] * (n - 1) + [3.0], (1, 1, 1), 4.0)
    s.set_projector(ntrace.PARALLEL, [0] * (n - 1) + [10], [0] * (n - 1) + [-1], np.eye(n)[: n - 1], 0.5, [8] * (n - 1))
    s.build(host_only=True)
    return s


@pytest.mark.parametrize("n,negative", [(3, False), (4, True), (5, False)])
def test_obj_mesh_equals_array_mesh(tmp_path, n, negative):
    from math_b200 import scenes

    v, f = scenes.sphere_hull(n, 200, seed=n)
    path = tmp_path / f"m.obj{n if n > 3 else ''}"
    _write_obj(path, v, f, negative=negative)
    a = _scene_from(n, lambda s: s.add_mesh(v, f))
    b = _scene_from(n, lambda s: s.add_obj_file(path))
    ia, ib = a.mesh_info(0), b.mesh_info(0)
    for k in ("facet_count", "node_count", "leaf_count", "index_count", "max_depth"):
        assert ia[k] == ib[k], k
    ta, tb = a.tree_export(0), b.tree_export(0)
    for k in ta:
        assert np.array_equal(ta[k], tb[k]), k


def test_obj_polygons_split_into_fans_and_normals(tmp_path):
    from math_b200 import ntrace

    # a cube of quads: 6 faces -> 12 triangles, each quad corner with its normal
    verts = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float32) - 0.5
    quads = [[0, 1, 3, 2], [4, 6, 7, 5], [0, 4, 5, 1], [2, 3, 7, 6], [0, 2, 6, 4], [1, 5, 7, 3]]
    normals = verts / np.linalg.norm(verts, axis=1, keepdims=True)
    lines = ["v " + " ".join(map(str, v)) for v in verts] + ["vn " + " ".join(map(str, v)) for v in normals]
    lines += ["f " + " ".join(f"{i + 1}//{i + 1}" for i in q) for q in quads]
    path = tmp_path / "cube.obj"
    path.write_text("\n".join(lines) + "\n")
    s = _scene_from(3, lambda sc: sc.add_obj_file(path))
    assert s.mesh_info(0)["facet_count"] == 12
    # the file's errors are reported with the file position
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nf 1 2\n")
    s2 = ntrace.Scene(3)
    with pytest.raises(ntrace.NtraceError, match="bad.obj:3"):
        s2.add_obj_file(bad)
    missing = ntrace.Scene(3)
    with pytest.raises(ntrace.NtraceError):
        missing.add_obj_file(tmp_path / "none.obj")


@pytest.mark.gpu
def test_obj_scene_renders_like_array_scene(require_gpu, tmp_path):
    from math_b200 import scenes

    spec = scenes.config("n4_small")
    path = tmp_path / "m.obj4"
    _write_obj(path, spec["verts"], spec["facets"])
    a = scenes.build_scene(spec)
    b_spec = dict(spec, verts=None, facets=None)
    from math_b200 import ntrace

    b = ntrace.Scene(4)
    b.add_obj_file(path, color=spec["mesh_color"], diffuse=spec["mesh_diffuse"])
    fl = spec["floor"]
    b.add_parallelotope(fl["org"], fl["edges"], color=fl["color"], diffuse=fl["diffuse"])
    L = spec["light"]
    b.add_point_light(L["pos"], L["color"], L["unit"])
    P = spec["projector"]
    b.set_projector(P["kind"], P["org"], P["dir"], P["axes"], P["param"], P["screen"])
    bg = spec["bg"]
    b.set_background(bg["color"], bg["light"], bg["light_color"])
    b.build()
    for s in (a, b):
        s.render(spec["spp"], max_depth=spec["max_depth"], seed=2)
    ia, _ = a.image()
    ib, _ = b.image()
    assert np.abs(ia - ib).max() <= 1e-6 * max(1.0, np.abs(ia).max())
    del b_spec
