"""The CPU restatement (oracle/ntrace_oracle.c) pinned against the reference and its known answers.

Pins, in the order the reference's own tests establish them:
  * golden closest-hit fixtures produced by the compiled reference (tests/golden/make_golden.py): the
    oracle's Mesh<N,double> and Mesh<N,float> must give the same facet index and the same distance,
    bit for bit, for every ray (the query of src/painter/shapes/test/test_mesh.cpp:139-152);
  * the reference tree's box and facet-reference counts;
  * cosine_sphere_coefficient's exact values (src/painter/coefficient/cosine_sphere.cpp:35-49);
  * the stratified sampler's effective sample counts (src/painter/sampling/sampler.h:31-52);
  * Philox4x32-10 against the published Random123 known-answer vectors;
  * the cosine-weighted hemisphere histogram (src/painter/sampling/test/test_sphere.cpp:69-123);
  * the two-hit invariant on a closed sphere mesh (src/painter/shapes/test/test_mesh.cpp:106-223).
"""

import math

import numpy as np
import pytest

from conftest import GOLDEN


_MESHES: dict = {}


def _fixture_mesh(port, n, dbl):
    key = (n, dbl)
    if key not in _MESHES:
        g = np.load(GOLDEN / f"closest_n{n}.npz")
        _MESHES[key] = (g, port.mesh(n, g["verts"], g["facets"], dbl=dbl))
    return _MESHES[key]


@pytest.mark.parametrize("n", [3, 4, 5, 6])
@pytest.mark.parametrize("dbl", [True, False])
def test_closest_hit_matches_reference_fixture(port, n, dbl):
    g, mesh = _fixture_mesh(port, n, dbl)
    facet, t, _ = port.trace(mesh, g["org"], g["dir"])
    ref_facet = g["facet64"] if dbl else g["facet32"]
    ref_t = g["t64"] if dbl else g["t32"]
    assert np.array_equal(facet, ref_facet)
    assert np.array_equal(t, ref_t)


@pytest.mark.parametrize("n", [3, 4, 5, 6])
@pytest.mark.parametrize("dbl", [True, False])
def test_tree_matches_reference_counts(port, n, dbl):
    g, mesh = _fixture_mesh(port, n, dbl)
    key = "64" if dbl else "32"
    tree = port.tree(mesh)
    assert len(tree["first_child"]) == int(g["boxes" + key])
    assert len(tree["indices"]) == int(g["indices" + key])


def test_cosine_sphere_coefficient_known_answers(port):
    # cosine_sphere.cpp:35-49
    expect = {2: math.pi / 2, 3: 2.0, 4: 3 * math.pi / 4, 5: 8.0 / 3, 6: 15 * math.pi / 16, 7: 16.0 / 5,
              8: 35 * math.pi / 32, 9: 128.0 / 35, 10: 315 * math.pi / 256, 15: 2048.0 / 429,
              20: 230945 * math.pi / 131072}
    for n, v in expect.items():
        assert port.cosine_sphere_coefficient(n) == pytest.approx(v, rel=1e-15)


def test_effective_samples_per_pixel(port):
    # k = floor or ceil of spp^(1/(n-1)), the first whose power reaches spp
    assert port.effective_spp(3, 16) == 16
    assert port.effective_spp(4, 16) == 27
    assert port.effective_spp(5, 16) == 16
    assert port.effective_spp(5, 4) == 16
    assert port.effective_spp(4, 4) == 8
    assert port.effective_spp(3, 65536) == 65536
    assert port.effective_spp(4, 65536) == 68921
    assert port.effective_spp(5, 65536) == 65536
    assert port.effective_spp(4, 4096) == 4096
    assert port.effective_spp(6, 1) == 1


def test_philox_known_answers(port):
    # Random123 kat_vectors, philox4x32 with 10 rounds
    assert list(port.philox(0, [0, 0, 0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(port.philox(0xFFFFFFFFFFFFFFFF, [0xFFFFFFFF] * 4)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    key = 0xA4093822 | (0x299F31D0 << 32)
    assert list(port.philox(key, [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344])) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("n", [3, 4, 5, 6])
def test_cosine_hemisphere_histogram(port, n):
    """cos(theta) of the sampled directions follows the cosine-weighted density (test_sphere.cpp)."""
    rng = np.random.default_rng(n)
    normal = rng.standard_normal(n)
    normal /= np.linalg.norm(normal)
    count = 40000
    cosines = np.empty(count)
    for i in range(count):
        d = port.cosine_hemisphere(n, normal, seed=7, path=i, stream=1)
        assert d is not None
        assert abs(np.linalg.norm(d) - 1.0) < 1e-12
        cosines[i] = d @ normal
    assert cosines.min() >= 0.0
    # The reference's test normalises the histogram of cos(theta) by its largest bucket and requires
    # it to equal cos(theta) (test_sphere.cpp:69-123): the density of c = cos(theta) is 2c in every
    # dimension (the radial rescale |v|^(n/2 - 1.5) of sphere.h:98-103 makes it so for n >= 4).
    bins = 20
    hist, edges = np.histogram(cosines, bins=bins, range=(0.0, 1.0), density=True)
    centres = (edges[:-1] + edges[1:]) / 2
    expect = 2.0 * centres
    assert np.max(np.abs(hist - expect)) < 0.05 * 2.0


@pytest.mark.parametrize("n,points", [(3, 600), (4, 300)])
def test_two_hit_invariant_on_sphere_mesh(port, n, points):
    """Rays from outside a closed sphere mesh hit it twice and not a third time (test_mesh.cpp:106-223)."""
    from math_b200 import scenes

    verts, facets = scenes.sphere_hull(n, points, seed=5)
    mesh = port.mesh(n, verts, facets, dbl=True)
    rng = np.random.default_rng(3)
    count = 3000
    d = rng.standard_normal((count, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = (2.0 * d + 0.0099).astype(np.float32)
    dirs = (-d).astype(np.float32)
    # the ray origins cross the interface as float32: offset by 100 float32 epsilons of the
    # coordinate scale (test_mesh.cpp:79 uses 100 epsilons of the mesh's own type)
    offset = 100 * float(np.finfo(np.float32).eps) * 2.0
    f1, t1, _ = port.trace(mesh, org, dirs)
    unit = dirs.astype(np.float64) / np.linalg.norm(dirs.astype(np.float64), axis=1, keepdims=True)
    o2 = (org + unit * (t1 + offset)[:, None]).astype(np.float32)
    f2, t2, _ = port.trace(mesh, o2, dirs)
    o3 = (o2 + unit * (t2 + offset)[:, None]).astype(np.float32)
    f3, _, _ = port.trace(mesh, o3, dirs)
    errors = (f1 < 0) | (f2 < 0) | (f3 >= 0)
    assert errors.mean() <= 0.0005 + 2.0 / count


def test_port_matches_reference_closest_hits(port, reference):
    """Beyond the fixtures: a fresh mesh and ray set, oracle against the reference library."""
    from math_b200 import scenes

    verts, facets = scenes.sphere_hull(4, 500, seed=21)
    rng = np.random.default_rng(4)
    d = rng.standard_normal((4000, 4))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = (1.7 * d).astype(np.float32)
    dirs = (-d + 0.1 * rng.standard_normal((4000, 4))).astype(np.float32)
    for dbl in (True, False):
        f_p, t_p, _ = port.trace(port.mesh(4, verts, facets, dbl=dbl), org, dirs)
        f_r, t_r = reference.trace(reference.mesh(4, verts, facets, dbl=dbl), org, dirs)
        assert np.array_equal(f_p, f_r)
        assert np.array_equal(t_p, t_r)


def test_port_radiance_matches_reference_statistically(port):
    """The oracle's painter (Philox stream) against the reference's own paint() image (mt19937 stream):
    independent noise, so the difference must be of the size of the reference's run-to-run noise."""
    from math_b200 import scenes

    g = np.load(GOLDEN / "radiance_n3.npz")
    spec = scenes.make_spec(3, g["verts"], g["facets"], screen=int(g["screen"]), spp=int(g["spp"]),
                            max_depth=int(g["max_depth"]))
    img, _ = port.paint(spec, dbl=True, threads=4)
    a, b = g["image_a"], g["image_b"]
    noise = np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())
    diff = np.sqrt(((img - a) ** 2).sum() / (a ** 2).sum())
    assert diff < 1.5 * noise


def test_port_smooth_normal_radiance_matches_reference_statistically(port):
    """Vertex normals of every NormalType with smooth_normal set (shading-normal interpolation and the
    smooth-normal shadow branch, painter.cpp:238-284): the oracle against the reference's paint()."""
    from math_b200 import scenes

    g = np.load(GOLDEN / "radiance_n3_smooth.npz")
    spec = scenes.make_spec(3, g["verts"], g["facets"], screen=int(g["screen"]), spp=int(g["spp"]),
                            max_depth=int(g["max_depth"]), extent=float(g["extent"]))
    spec["normals"] = g["normals"]
    spec["smooth_normal"] = True
    img, _ = port.paint(spec, dbl=True, threads=4)
    a, b = g["image_a"], g["image_b"]
    noise = np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())
    diff = np.sqrt(((img - a) ** 2).sum() / (a ** 2).sum())
    assert diff < 1.5 * noise, (diff, noise)
    # the flat-shaded image is far outside that noise: the test sees the smooth shading
    flat = dict(spec, smooth_normal=False)
    img_flat, _ = port.paint(flat, dbl=True, threads=4)
    assert np.sqrt(((img_flat - a) ** 2).sum() / (a ** 2).sum()) > 5 * noise
