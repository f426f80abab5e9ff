"""2^n-tree built on the GPU (nt_build_opts.tree_on_gpu): the same tree as the host build, box for
box and reference for reference (the device runs the host's box-simplex overlap code), hence the
same images."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _build(spec, **kw):
    from math_b200 import ntrace

    n = spec["n"]
    s = ntrace.Scene(n)
    s.add_mesh(spec["verts"], spec["facets"])
    fl = spec["floor"]
    s.add_parallelotope(fl["org"], fl["edges"])
    L = spec["light"]
    s.add_point_light(L["pos"], L["color"], L["unit"])
    P = spec["projector"]
    s.set_projector(P["kind"], P["org"], P["dir"], P["axes"], P["param"], P["screen"])
    s.build(**kw)
    return s


def _same_tree(a, b):
    ia, ib = a.mesh_info(0), b.mesh_info(0)
    for k in ("node_count", "leaf_count", "index_count", "max_depth"):
        assert ia[k] == ib[k], (k, ia[k], ib[k])
    ta, tb = a.tree_export(0), b.tree_export(0)
    for k in ta:
        assert np.array_equal(ta[k], tb[k]), k


@pytest.mark.parametrize("name", ["n3_small", "n4_small", "n5_small", "n6_small"])
def test_gpu_tree_equals_host_tree(require_gpu, name):
    from math_b200 import scenes

    spec = scenes.config(name)
    _same_tree(_build(spec, host_only=True), _build(spec, tree_on_gpu=True))


@pytest.mark.parametrize("n,points", [(3, 20000), (4, 5000), (5, 1000)])
def test_gpu_tree_equals_host_tree_larger(require_gpu, n, points):
    from math_b200 import scenes

    v, f = scenes.sphere_hull(n, points, seed=11)
    spec = scenes.make_spec(n, v, f, screen=8, spp=1)
    a = _build(spec, host_only=True)
    b = _build(spec, tree_on_gpu=True)
    _same_tree(a, b)
    assert b.mesh_info(0)["index_count"] >= len(f)


def test_gpu_tree_scene_renders_like_host_tree_scene(require_gpu):
    from math_b200 import scenes

    spec = scenes.config("n4_small")
    a = scenes.build_scene(spec)
    b = scenes.build_scene(spec, tree_on_gpu=True)
    for s in (a, b):
        s.render(spec["spp"], max_depth=spec["max_depth"], seed=8)
    ia, _ = a.image()
    ib, _ = b.image()
    assert np.abs(ia - ib).max() <= 1e-6 * max(1.0, np.abs(ia).max())
