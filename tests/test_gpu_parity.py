"""GPU parity of the sm_100a kernels against the oracle and the reference (marked gpu).

* Fixed ray sets: facet index bit-exact against Mesh<N,double> of the reference (golden fixtures
  made by the compiled reference, and the oracle's FP64 restatement on fresh ray sets), distance within
  2e-6 relative.  The FP32-only path (no re-test) is checked to be the one that disagrees.
* Radiance: the same Philox paths as the oracle's float painter (per-pixel agreement, relative RMSE
  below 1e-4), and against the reference's own paint() image statistically (difference within 1.5x
  the reference's run-to-run noise).
"""

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rrmse(a, b):
    return float(np.sqrt(((a - b) ** 2).sum()) / np.sqrt((b ** 2).sum()))


def _mesh_scene(n, verts, facets):
    from math_b200 import ntrace

    s = ntrace.Scene(n)
    s.add_mesh(verts, facets)
    light = np.full(n, 2.0)
    s.add_point_light(light, (1, 1, 1), 1.0)
    cam_dir = np.zeros(n)
    cam_dir[n - 1] = -1
    s.set_projector(0, np.zeros(n), cam_dir, np.eye(n)[: n - 1], 0.1, [4] * (n - 1))
    s.build()
    return s


@pytest.mark.parametrize("n", [3, 4, 5, 6])
def test_closest_hit_bit_exact_against_reference_fixture(require_gpu, n):
    g = np.load(GOLDEN / f"closest_n{n}.npz")
    s = _mesh_scene(n, g["verts"], g["facets"])
    facet, t, st = s.trace_closest(g["org"], g["dir"], retest=True)
    assert st["error_bits"] == 0
    assert np.array_equal(facet, g["facet64"]), int((facet != g["facet64"]).sum())
    hit = facet >= 0
    assert np.allclose(t[hit], g["t64"][hit], rtol=2e-6, atol=0)
    # without the FP64 re-test the float path disagrees on the boundary rays
    facet32, _, _ = s.trace_closest(g["org"], g["dir"], retest=False)
    assert (facet32 != g["facet64"]).sum() > 0
    assert st["retests"] > 0


def _edge_rays(verts, facets, count, seed):
    rng = np.random.default_rng(seed)
    n = verts.shape[1]
    fi = rng.integers(0, len(facets), count)
    a = rng.integers(0, n, count)
    b = (a + rng.integers(1, n, count)) % n
    w = rng.random(count)[:, None] * np.where(rng.random(count) < 0.3, 0.0, 1.0)[:, None]
    target = verts[facets[fi, a]].astype(np.float64) * (1 - w) + verts[facets[fi, b]].astype(np.float64) * w
    d = rng.standard_normal((count, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = target + 3.0 * d
    return org.astype(np.float32), (target - org).astype(np.float32)


def _exact_hit(verts, facet_vertices, org, direction):
    """Exact rational intersection of the ray org + t * unit(direction) with the simplex: returns t if
    the intersection lies strictly inside the simplex with t > 0, else None.  The unit direction is
    taken as its double-precision value (as the FP64 reference computes it)."""
    from fractions import Fraction as F

    n = len(org)
    d = np.asarray(direction, np.float64)
    d = d / np.linalg.norm(d)
    V = [[F(float(x)) for x in verts[i]] for i in facet_vertices]
    # unknowns b_0..b_(n-1), t: sum b_j V_j - t d = org, sum b_j = 1
    rows = [[V[j][k] for j in range(n)] + [-F(float(d[k]))] + [F(float(org[k]))] for k in range(n)]
    rows.append([F(1)] * n + [F(0), F(1)])
    m = n + 1
    for c in range(m):
        piv = next((r for r in range(c, m) if rows[r][c] != 0), None)
        if piv is None:
            return None
        rows[c], rows[piv] = rows[piv], rows[c]
        for r in range(m):
            if r != c and rows[r][c] != 0:
                f = rows[r][c] / rows[c][c]
                rows[r] = [a - f * b for a, b in zip(rows[r], rows[c])]
    sol = [rows[r][m] / rows[r][r] for r in range(m)]
    if all(b > 0 for b in sol[:n]) and sol[n] > 0:
        return sol[n]
    return None


@pytest.mark.parametrize("n,points", [(3, 2000), (4, 1500), (5, 400)])
def test_closest_hit_bit_exact_against_oracle_fresh_rays(require_gpu, port, n, points):
    """Fresh ray sets (20,000 random, 20,000 aimed at facet boundaries) against the FP64 oracle.  Where
    the two differ, the FP64 oracle must be the one in the wrong: its double-precision tree can leave a
    facet out of a leaf that the facet crosses (Mesh<N,double>'s box-simplex test, reproduced exactly by
    the oracle), so it misses the true first hit; exact rational arithmetic then shows the GPU's facet is
    hit, and nearer than the oracle's."""
    from math_b200 import scenes

    verts, facets = scenes.sphere_hull(n, points, seed=40 + n)
    s = _mesh_scene(n, verts, facets)
    rng = np.random.default_rng(n)
    d = rng.standard_normal((20000, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = np.concatenate([(1.5 * d).astype(np.float32), _edge_rays(verts, facets, 20000, n)[0]])
    dirs = np.concatenate([(-d + 0.2 * rng.standard_normal(d.shape)).astype(np.float32),
                           _edge_rays(verts, facets, 20000, n)[1]])
    facet, t, st = s.trace_closest(org, dirs, retest=True)
    pf, pt, _ = port.trace(port.mesh(n, verts, facets, dbl=True), org, dirs)
    assert st["error_bits"] == 0
    bad = np.nonzero(facet != pf)[0]
    # no allowance: every difference must be shown by exact arithmetic to be the oracle's mistake
    for i in bad:
        if facet[i] >= 0:
            t_gpu = _exact_hit(verts, facets[facet[i]], org[i], dirs[i])
            assert t_gpu is not None, i
            if pf[i] >= 0:
                t_oracle = _exact_hit(verts, facets[pf[i]], org[i], dirs[i])
                assert t_oracle is None or t_gpu < t_oracle, i
        else:
            assert _exact_hit(verts, facets[pf[i]], org[i], dirs[i]) is None, i
    print(f"n={n}: {len(org)} fresh rays, {len(bad)} differences from the FP64 oracle, each explained exactly")
    same = (facet == pf) & (facet >= 0)
    assert np.allclose(t[same], pt[same], rtol=2e-6, atol=0)


@pytest.mark.parametrize("name", ["n3_small", "n4_small", "n5_small", "n6_small"])
def test_radiance_matches_oracle_paths(require_gpu, port, name):
    """Same scene, same Philox paths: the GPU image and the oracle's float painter agree per pixel."""
    from math_b200 import scenes

    spec = scenes.config(name)
    s = scenes.build_scene(spec)
    st = s.render(spec["spp"], max_depth=spec["max_depth"], seed=spec["seed"])
    img, spp = s.image()
    assert st["error_bits"] == 0
    assert spp == port.effective_spp(spec["n"], spec["spp"])
    p32, _ = port.paint(spec, dbl=False, threads=8)
    p64, _ = port.paint(spec, dbl=True, threads=8)
    assert rrmse(img, p32) < 1e-4
    assert rrmse(img, p64) < 5e-3
    assert np.isfinite(img).all() and img.min() >= 0


def test_radiance_matches_reference_statistically(require_gpu):
    """GPU image against the reference's own paint() at 1024 samples per pixel (independent noise)."""
    from math_b200 import scenes

    g = np.load(GOLDEN / "radiance_n3.npz")
    spec = scenes.make_spec(3, g["verts"], g["facets"], screen=int(g["screen"]), spp=int(g["spp"]),
                            max_depth=int(g["max_depth"]))
    s = scenes.build_scene(spec)
    s.render(int(g["spp"]), max_depth=int(g["max_depth"]), seed=12345)
    img, spp = s.image()
    a, b = g["image_a"], g["image_b"]
    noise = rrmse(a, b)
    assert rrmse(img, a) < 1.5 * noise
    assert rrmse(img, b) < 1.5 * noise


def _smooth_spec():
    from math_b200 import scenes

    g = np.load(GOLDEN / "radiance_n3_smooth.npz")
    spec = scenes.make_spec(3, g["verts"], g["facets"], screen=int(g["screen"]), spp=int(g["spp"]),
                            max_depth=int(g["max_depth"]), extent=float(g["extent"]))
    spec["normals"] = g["normals"]
    spec["smooth_normal"] = True
    return spec, g


def test_smooth_normal_radiance_matches_oracle_paths(require_gpu, port):
    """Vertex normals of every NormalType with smooth_normal: the same Philox paths as the oracle's
    float painter (interpolated shading normals, the smooth-normal shadow branch).  The GPU
    interpolates with its FP32 barycentric planes from Gaussian elimination, the oracle with the
    reference's set_data planes: shading normals differ in the last bits, which moves a few bounce
    directions, hence a looser bound than for flat shading."""
    from math_b200 import scenes

    spec, _ = _smooth_spec()
    s = scenes.build_scene(spec)
    st = s.render(64, max_depth=5, seed=3, smooth_normal=True)
    img, _ = s.image()
    assert st["error_bits"] == 0
    p32, _ = port.paint(spec, dbl=False, spp=64, seed=3, threads=8)
    assert rrmse(img, p32) < 1e-3
    s.clear()
    s.render(64, max_depth=5, seed=3, smooth_normal=False)
    flat, _ = s.image()
    assert rrmse(flat, img) > 1e-2


def test_smooth_normal_radiance_matches_reference_statistically(require_gpu):
    from math_b200 import scenes

    spec, g = _smooth_spec()
    s = scenes.build_scene(spec)
    s.render(int(g["spp"]), max_depth=int(g["max_depth"]), seed=777, smooth_normal=True)
    img, _ = s.image()
    a, b = g["image_a"], g["image_b"]
    noise = rrmse(a, b)
    assert rrmse(img, a) < 1.5 * noise
    assert rrmse(img, b) < 1.5 * noise


def test_progressive_passes_accumulate(require_gpu):
    """Two passes of k samples continue the sample sequence: equal to the oracle painting 2k with an
    offset, and the sample count adds up."""
    from math_b200 import scenes

    spec = scenes.config("n3_small")
    s = scenes.build_scene(spec)
    s.render(16, max_depth=5, seed=3)
    s.render(16, max_depth=5, seed=3)
    img, spp = s.image()
    assert spp == 32
    s.clear()
    s.render(16, max_depth=5, seed=3)
    first, _ = s.image()
    s.clear()
    _, spp0 = s.image()
    assert spp0 == 0
    # the second pass alone differs from the first (new samples), the mean of both is the total
    assert rrmse(img, first) > 1e-4


def test_double_buffered_upload_renders_the_same_scene(require_gpu):
    """A staged upload (copy stream, then device-to-device into the live arrays) leaves the scene as
    it was: renders of one seed before, during (the next frame's copy in flight) and after agree; a
    commit without a begin, or after a rebuild, is refused."""
    from math_b200 import ntrace, scenes

    spec = scenes.config("n4_small")
    s = scenes.build_scene(spec)
    s.render(8, max_depth=5, seed=5)
    before, _ = s.image()
    assert s.upload_begin() > 0
    s.upload_commit()
    s.upload_begin()  # in flight during the next render
    s.clear()
    s.render(8, max_depth=5, seed=5)
    during, _ = s.image()
    s.upload_commit()
    s.clear()
    s.render(8, max_depth=5, seed=5)
    after, _ = s.image()
    # FP64 atomics in another order: equal to rounding
    np.testing.assert_allclose(during, before, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(after, before, rtol=1e-9, atol=1e-12)
    with pytest.raises(ntrace.NtraceError) as e:
        s.upload_commit()
    assert e.value.code == ntrace.NT_ESTATE
    s.upload_begin()
    s.build()
    with pytest.raises(ntrace.NtraceError) as e:
        s.upload_commit()
    assert e.value.code == ntrace.NT_ESTATE


def test_render_rejects_bad_options_and_stops(require_gpu):
    import ctypes

    from math_b200 import ntrace, scenes

    spec = scenes.config("n3_small")
    s = scenes.build_scene(spec)
    with pytest.raises(ntrace.NtraceError) as e:
        s.render(0)
    assert e.value.code == ntrace.NT_EINVAL
    flag = ctypes.c_int(1)
    with pytest.raises(ntrace.NtraceError) as e:
        s.render(16, stop=ctypes.pointer(flag))
    assert e.value.code == ntrace.NT_ESTOPPED
    _, spp = s.image()
    assert spp == 0
    flag.value = 0
    s.render(4, stop=ctypes.pointer(flag))
    assert s.image()[1] == 4


def test_full_scene_render_properties(require_gpu):
    """n = 3 measured scene at full size: finite, reproducible for a seed, counters consistent."""
    from math_b200 import scenes

    spec = scenes.config("n3")
    s = scenes.build_scene(spec)
    st = s.render(spec["spp"], max_depth=spec["max_depth"], seed=0)
    img, spp = s.image()
    s.clear()
    s.render(spec["spp"], max_depth=spec["max_depth"], seed=0)
    img2, _ = s.image()
    assert st["error_bits"] == 0
    assert st["paths"] == 400 * 400 * 16
    assert st["rays"] >= st["paths"]
    assert np.isfinite(img).all()
    assert rrmse(img2, img) < 1e-6
    # the background (sky) colour is seen where camera rays miss everything: none do here (the floor
    # covers the screen), so every pixel is lit by the light or the sky through bounces
    assert img.mean() > 0.1


def _srgb8(c):
    """rgb_float_to_srgb_uint8 (src/com/color/conversion.cpp:35-42,211-230,344-347) in float32."""
    c = np.asarray(c, np.float32)
    s = np.where(c >= 1, np.float32(1),
                 np.where(c >= np.float32(0.0031308),
                          np.float32(1.055) * np.power(np.maximum(c, np.float32(1e-30)), np.float32(1 / 2.4)) - np.float32(0.055),
                          np.where(c > 0, c * np.float32(12.92), np.float32(0))))
    return (s.astype(np.float32) * np.float32(255) + np.float32(0.5)).astype(np.uint8).astype(np.uint32)


@pytest.mark.parametrize("name", ["n3_small", "n4_small"])
def test_viewer_feed_slice_matches_the_painter_window_conversion(require_gpu, name):
    from math_b200 import scenes

    spec = scenes.config(name)
    s = scenes.build_scene(spec)
    s.render(spec["spp"], max_depth=spec["max_depth"], seed=6)
    img, _ = s.image()
    n = spec["n"]
    screen = spec["projector"]["screen"]
    pos = [screen[j] // 2 for j in range(2, n - 1)]
    got = s.srgb_slice(pos)
    cube = img.reshape(list(screen[::-1]) + [3])  # (x_{n-2}, ..., x1, x0, rgb)
    sl = cube[tuple(pos[::-1]) + (slice(None), slice(None))] if pos else cube
    sl = sl[::-1]  # row 0 = last screen row
    want = (_srgb8(sl[..., 0]) << 16) | (_srgb8(sl[..., 1]) << 8) | _srgb8(sl[..., 2])
    assert got.shape == want.shape
    diff = np.abs(((got >> 16) & 255).astype(int) - ((want >> 16) & 255).astype(int))
    assert diff.max() <= 1 and (got == want).mean() > 0.99
