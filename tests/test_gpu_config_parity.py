"""Parity at the measured configurations' scale against the reference itself (marked gpu).

* Fixed ray sets through the measured meshes (20,480 / 675,461 / 1,541,774 facets at n = 3, 4, 5):
  the facet index of every ray equals Mesh<N,double>'s (tests/golden/config_rays_*.npz, made by the
  compiled reference), except where exact rational arithmetic shows the reference to be the one in the
  wrong (its double-precision tree leaves the true first facet out of the leaf the hit lies in).
* Converged radiance: 1,024 seeded pixels of each configuration scene (and a six-dimensional one) at
  65,536 samples per pixel (68,921 at n = 4, 100,000 at n = 6) against the reference's
  paint<N,double>() at the same sample count (tests/golden/config_radiance_*.npz): relative RMSE at
  most 1e-3 (the criterion stated for the path), and no bias in the mean over the pixels beyond 4.5
  standard errors.
* Whole images of small n = 4, 5, 6 scenes at 1,024 samples per pixel against two reference images:
  the squared difference per pixel is what the noise of the three renders predicts, and the mean shows
  no bias.
* Sample ranges: passes at explicit sample offsets (one rank's share of a frame) add up to the
  progressive passes of one scene; a pixel-list pass traces the same paths as the whole frame.
"""

from __future__ import annotations

import hashlib
from functools import lru_cache

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rrmse(a, b):
    return float(np.sqrt(((a - b) ** 2).sum()) / np.sqrt((b ** 2).sum()))


def digest(verts, facets) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(verts, np.float32).tobytes())
    h.update(np.ascontiguousarray(facets, np.int32).tobytes())
    return h.hexdigest()


@lru_cache(maxsize=None)
def config_spec(name: str) -> dict:
    from math_b200 import scenes

    return scenes.config(name)


_SCENES: dict = {}


def config_scene(name: str):
    """The configuration scene, built once per session (trees on the GPU: the same trees, box for
    box, as the host build)."""
    from math_b200 import scenes

    if name not in _SCENES:
        _SCENES.clear()  # one large scene at a time on the device
        _SCENES[name] = scenes.build_scene(config_spec(name), tree_on_gpu=True)
    return _SCENES[name]


def _check_mesh(g, spec):
    assert int(g["facet_count"]) == len(spec["facets"]) and int(g["vertex_count"]) == len(spec["verts"])
    assert str(g["digest"]) == digest(spec["verts"], spec["facets"]), "the configuration mesh changed"


@pytest.mark.parametrize("name", ["n3", "n4", "n5"])
def test_config_mesh_closest_hits_match_reference(require_gpu, name):
    from test_gpu_parity import _exact_hit

    g = np.load(GOLDEN / f"config_rays_{name}.npz")
    spec = config_spec(name)
    _check_mesh(g, spec)
    s = config_scene(name)
    org, dirs, want = g["org"], g["dir"], g["facet64"]
    facet, t, st = s.trace_closest(org, dirs, retest=True)
    assert st["error_bits"] == 0
    verts, facets = spec["verts"], spec["facets"]
    bad = np.nonzero(facet != want)[0]
    for i in bad:
        # each difference must be the reference's mistake, shown exactly
        if facet[i] >= 0:
            t_gpu = _exact_hit(verts, facets[facet[i]], org[i], dirs[i])
            assert t_gpu is not None, (name, int(i), int(facet[i]), int(want[i]))
            if want[i] >= 0:
                t_ref = _exact_hit(verts, facets[want[i]], org[i], dirs[i])
                assert t_ref is None or t_gpu < t_ref, (name, int(i))
        else:
            assert _exact_hit(verts, facets[want[i]], org[i], dirs[i]) is None, (name, int(i))
    same = (facet == want) & (facet >= 0)
    assert np.allclose(t[same], g["t64"][same], rtol=2e-6, atol=0)
    print(f"{name}: {len(org)} rays, {int((want >= 0).sum())} hits, {len(bad)} differences (each explained "
          f"exactly), {st['retests']} FP64 re-tests")
    # without the FP64 re-test the float path disagrees somewhere on these rays
    facet32, _, _ = s.trace_closest(org, dirs, retest=False)
    assert (facet32 != want).sum() >= len(bad)


@pytest.mark.parametrize("name", ["n3", "n4", "n5", "n6"])
def test_converged_radiance_matches_reference(require_gpu, name):
    g = np.load(GOLDEN / f"config_radiance_{name}.npz")
    spec = config_spec(name)
    _check_mesh(g, spec)
    s = config_scene(name)
    spp = int(g["spp"])
    img, st = s.render_pixels(g["pixels"], spp, max_depth=int(g["max_depth"]), seed=424242)
    assert st["error_bits"] == 0 and st["spp_effective"] == int(g["spp_effective"])
    a, b = g["image_a"].astype(np.float64), g["image_b"].astype(np.float64)
    e_a, e_b, noise = rrmse(img, a), rrmse(img, b), rrmse(a, b)
    print(f"{name}: {len(img)} pixels x {int(g['spp_effective'])} spp: relative RMSE vs reference "
          f"{e_a:.2e} / {e_b:.2e} (reference vs itself {noise:.2e})")
    assert e_a <= 1e-3 and e_b <= 1e-3
    # the mean over the pixels: the GPU and the reference's average differ by noise only
    from test_gpu_interfaces import bias_z

    z = bias_z(img, a, b)
    print(f"{name}: bias of the pixel sum, standard score {z:.2f}")
    assert abs(z) < 4.5, z


@pytest.mark.parametrize("name", ["n4_small", "n5_small", "n6_small"])
def test_small_images_match_reference_statistically(require_gpu, name):
    from math_b200 import scenes

    g = np.load(GOLDEN / f"radiance_{name}.npz")
    spec = scenes.config(name)
    _check_mesh(g, spec)
    s = scenes.build_scene(spec)
    s.render(int(g["spp"]), max_depth=int(g["max_depth"]), seed=99)
    img, _ = s.image()
    a, b = g["image_a"].astype(np.float64), g["image_b"].astype(np.float64)
    d2 = (a - b) ** 2 / 2  # per-pixel estimate of one render's noise variance
    ref = (a + b) / 2
    r = (img - ref) ** 2
    ratio = r.sum() / (1.5 * d2.sum())  # 1 if the GPU image has the reference's expected value
    from test_gpu_interfaces import bias_z

    z = bias_z(img, a, b)
    print(f"{name}: squared difference / predicted noise {ratio:.3f}, bias z {z:.2f}")
    assert 0.7 < ratio < 1.3
    assert abs(z) < 4.5


def test_sample_offset_ranges_add_up_to_progressive_passes(require_gpu):
    """Two scenes rendering samples [0, k) and [k, 2k) (sample_offset; as two ranks would) sum to one
    scene's two progressive passes: the same paths."""
    from math_b200 import ntrace, scenes

    spec = scenes.config("n4_small")
    spp, depth = spec["spp"], spec["max_depth"]
    k = ntrace.effective_spp(4, spp)
    ra, rb, both = (scenes.build_scene(spec) for _ in range(3))
    ra.render(spp, max_depth=depth, seed=5, sample_offset=0)
    rb.render(spp, max_depth=depth, seed=5, sample_offset=k)
    both.render(spp, max_depth=depth, seed=5)
    both.render(spp, max_depth=depth, seed=5)
    a, na = ra.image()
    b, nb = rb.image()
    c, nc = both.image()
    assert na == nb == k and nc == 2 * k
    combined = (a.astype(np.float64) * k + b.astype(np.float64) * k) / (2 * k)
    assert rrmse(combined, c.astype(np.float64)) < 1e-6
    assert rrmse(a, b) > 1e-3  # the two ranges are different samples


def test_pixel_list_traces_the_frame_paths(require_gpu):
    from math_b200 import scenes

    spec = scenes.config("n3_small")
    s = scenes.build_scene(spec)
    s.render(spec["spp"], max_depth=5, seed=8)
    full, _ = s.image()
    rng = np.random.default_rng(3)
    lin = rng.choice(s.pixel_count, 300, replace=False)
    lin[:5] = lin[0]  # repeats are allowed
    sub, st = s.render_pixels(lin, spec["spp"], max_depth=5, seed=8)
    assert st["paths"] == 300 * 16
    np.testing.assert_allclose(sub, full[lin], rtol=2e-6, atol=1e-7)
    # a later sample range gives other samples of the same pixels
    later, _ = s.render_pixels(lin, spec["spp"], max_depth=5, seed=8, sample_offset=16)
    assert rrmse(later, full[lin]) > 1e-3
    # the accumulator was not touched
    again, n = s.image()
    assert n == 16 and np.array_equal(again, full)
