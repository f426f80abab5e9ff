"""Host side of the product library, without a GPU: the C ABI loads and exports what include/*.h
declares, the multithreaded float tree build reproduces the reference's Mesh<N,float> tree (as
restated by the oracle, itself pinned to the reference), and malformed scenes are rejected with the
documented status codes before anything is launched."""

import ctypes
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def _header_functions():
    text = "\n".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\*?\s+\**(nt_[a-z0-9_]+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    from math_b200 import ntrace

    lib = ctypes.CDLL(str(ntrace.LIB_PATH))
    names = _header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) >= set(ntrace.EXPORTED_SYMBOLS)


def test_library_scalar_helpers_match_oracle(port):
    from math_b200 import ntrace

    for n in (3, 4, 5, 6):
        assert ntrace.cosine_sphere_coefficient(n) == pytest.approx(port.cosine_sphere_coefficient(n), rel=1e-15)
        for spp in (1, 2, 4, 16, 27, 100, 4096, 65536):
            assert ntrace.effective_spp(n, spp) == port.effective_spp(n, spp)


def _host_scene(n, verts, facets):
    from math_b200 import ntrace

    s = ntrace.Scene(n)
    s.add_mesh(verts, facets)
    light = np.full(n, 2.0)
    s.add_point_light(light, (1, 1, 1), 1.0)
    axes = np.eye(n)[: n - 1]
    cam_dir = np.zeros(n)
    cam_dir[n - 1] = -1
    s.set_projector(0, np.zeros(n), cam_dir, axes, 0.1, [4] * (n - 1))
    s.build(host_only=True)
    return s


def _assert_same_tree(tree, ptree):
    nodes = tree["nodes"]
    assert len(nodes) == len(ptree["first_child"])
    leaf = nodes[:, 1] >= 0
    assert np.array_equal(leaf, ptree["first_child"] < 0)
    assert np.array_equal(nodes[~leaf, 0], ptree["first_child"][~leaf])
    for i in np.nonzero(leaf)[0]:
        a = ptree["indices"][ptree["offset"][i]:ptree["offset"][i + 1]]
        b = tree["indices"][nodes[i, 0]:nodes[i, 0] + nodes[i, 1]]
        assert np.array_equal(a, b), i
    assert tree["distance_from_facet"] == pytest.approx(ptree["distance_from_facet"], rel=0, abs=0)


@pytest.mark.parametrize("n", [3, 4, 5])
def test_float_tree_identical_to_oracle(port, n):
    g = np.load(GOLDEN / f"closest_n{n}.npz")
    s = _host_scene(n, g["verts"], g["facets"])
    tree = s.tree_export()
    ptree = port.tree(port.mesh(n, g["verts"], g["facets"], dbl=False))
    _assert_same_tree(tree, ptree)
    # level sizes: root size halved exactly at each level
    sizes = tree["level_sizes"]
    assert np.array_equal(sizes[1:], sizes[:-1] / 2)
    info = s.mesh_info()
    assert info["node_count"] == int(g["boxes32"])
    assert info["index_count"] == int(g["indices32"])


def test_float_tree_identical_to_oracle_icosphere(port):
    from math_b200 import scenes

    v, f = scenes.icosphere(3)
    s = _host_scene(3, v, f)
    _assert_same_tree(s.tree_export(), port.tree(port.mesh(3, v, f, dbl=False)))


def _code(fn):
    from math_b200 import ntrace

    with pytest.raises(ntrace.NtraceError) as e:
        fn()
    return e.value.code


def test_rejects_malformed_scenes():
    from math_b200 import ntrace
    from math_b200.ntrace import NT_EDEGENERATE, NT_EINVAL, NT_ESTATE

    assert _code(lambda: ntrace.Scene(2)) == NT_EINVAL
    assert _code(lambda: ntrace.Scene(7)) == NT_EINVAL

    s = ntrace.Scene(3)
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    f = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]], np.int32)
    bad = v.copy()
    bad[1, 1] = np.nan
    assert _code(lambda: s.add_mesh(bad, f)) == NT_EINVAL
    # building an empty scene, or rendering an unbuilt one
    assert _code(lambda: s.build(host_only=True)) == NT_EINVAL
    assert _code(lambda: s.render(4)) == NT_ESTATE
    # facet index out of range
    s2 = ntrace.Scene(3)
    s2.add_mesh(v, np.array([[0, 1, 9]], np.int32))
    s2.add_point_light((0, 0, 5), (1, 1, 1), 1.0)
    s2.set_projector(0, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (8, 8))
    assert _code(lambda: s2.build(host_only=True)) == NT_EINVAL
    # degenerate simplex: its normal is not finite (mesh_hyperplane_simplex.cpp:86-89)
    s3 = ntrace.Scene(3)
    s3.add_mesh(v, np.array([[0, 1, 2], [0, 0, 1]], np.int32))
    s3.add_point_light((0, 0, 5), (1, 1, 1), 1.0)
    s3.set_projector(0, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (8, 8))
    assert _code(lambda: s3.build(host_only=True)) == NT_EDEGENERATE
    # screen axes not orthogonal to the camera direction (projector.h:29-50)
    s4 = ntrace.Scene(3)
    s4.add_mesh(v, f)
    s4.add_point_light((0, 0, 5), (1, 1, 1), 1.0)
    s4.set_projector(0, (0, 0, 5), (0, 0.3, -1), np.eye(3)[:2], 0.1, (8, 8))
    assert _code(lambda: s4.build(host_only=True)) == NT_EINVAL
    # no light source
    s5 = ntrace.Scene(3)
    s5.add_mesh(v, f)
    s5.set_projector(0, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (8, 8))
    assert _code(lambda: s5.build(host_only=True)) == NT_EINVAL
    # a scene built for the host only has no device arrays: uploads are refused
    s6 = ntrace.Scene(3)
    s6.add_mesh(v, f)
    s6.add_point_light((0, 0, 5), (1, 1, 1), 1.0)
    s6.set_projector(0, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (8, 8))
    s6.build(host_only=True)
    assert _code(lambda: s6.upload()) == NT_ESTATE
    assert _code(lambda: s6.upload_begin()) == NT_ESTATE
    assert _code(lambda: s6.upload_commit()) == NT_ESTATE
    # bad screen size and unknown projector kind
    assert _code(lambda: s5.set_projector(0, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (0, 8))) == NT_EINVAL
    assert _code(lambda: s5.set_projector(5, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (8, 8))) == NT_EINVAL
    # a host-only build cannot render
    s4b = ntrace.Scene(3)
    s4b.add_mesh(v, f)
    s4b.add_point_light((0, 0, 5), (1, 1, 1), 1.0)
    s4b.set_projector(0, (0, 0, 5), (0, 0, -1), np.eye(3)[:2], 0.1, (8, 8))
    s4b.build(host_only=True)
    assert _code(lambda: s4b.render(4)) == NT_ESTATE
    assert _code(lambda: s4b.trace_closest(np.zeros((1, 3)), np.ones((1, 3)))) == NT_ESTATE
    # the error message is kept per thread
    assert b"host only" in ntrace.library().nt_last_error_message()
