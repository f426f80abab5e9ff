"""GPU coverage of every scene type the C ABI exports beyond the measured configurations (marked gpu).

Scenes (math_b200.scenes.interface_scene): a ConstantLight (lights/light_source.h:59-78), the
perspective and spherical projectors (projectors/projector.h:102-151,206-275), a hyperplane
parallelotope (space/hyperplane_parallelotope.h:25-104, visible_shapes.h:31-73), and two meshes, a
closed sphere beside an open bowl on the floor whose bounces start inside the bowl's root box, so
that the sorted early break of ray_intersection (space/ray_intersection.h:26-105) meets the root box's
exit distance.  Each is checked twice:

* against the C restatement on the same Philox paths (per-pixel agreement, relative RMSE < 1e-4);
* against the reference's own paint<N,double>() at 1,024 samples per pixel
  (tests/golden/radiance_iface_*.npz, two reference images with different seeds): the GPU image's
  squared difference from the reference mean is what the three renders' noise predicts (ratio within
  0.7-1.3), and the sum over the image shows no bias beyond 4.5 standard errors (noise per pixel over
  the channel sums: a pixel's channels come from the same paths).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

NAMES = ["constant_light_n4", "perspective_n4", "spherical_n5", "hplt_n4", "two_mesh_n3"]


def rrmse(a, b):
    return float(np.sqrt(((a - b) ** 2).sum()) / np.sqrt((b ** 2).sum()))


def bias_z(img, a, b, renders: int = 1) -> float:
    """Standard score of the difference between the sum of an image (the mean of `renders` renders)
    and the sum of the mean of two reference images a and b.  The colour channels of a pixel come from
    the same paths, so the noise is taken per pixel over the channel sums; pixels are independent."""
    x = np.asarray(img, np.float64).sum(axis=1)
    pa, pb = a.sum(axis=1), b.sum(axis=1)
    v = (pa - pb) ** 2 / 2  # one reference render's variance, per pixel
    return float((x - (pa + pb) / 2).sum() / np.sqrt((v / renders + v / 2).sum()))


@pytest.mark.parametrize("name", NAMES)
def test_interface_scene_matches_oracle_paths(require_gpu, port, name):
    from math_b200 import scenes

    spec = scenes.interface_scene(name)
    s = scenes.build_scene(spec)
    st = s.render(spec["spp"], max_depth=spec["max_depth"], seed=21)
    img, spp = s.image()
    assert st["error_bits"] == 0 and spp == port.effective_spp(spec["n"], spec["spp"])
    p32, _ = port.paint(spec, dbl=False, seed=21, threads=8)
    err = rrmse(img, p32)
    print(f"{name}: GPU vs the restatement on the same paths: relative RMSE {err:.2e}")
    assert err < 1e-4
    assert np.isfinite(img).all() and img.min() >= 0


@pytest.mark.parametrize("name", NAMES)
def test_interface_scene_matches_reference_statistically(require_gpu, name):
    from math_b200 import scenes

    g = np.load(GOLDEN / f"radiance_iface_{name}.npz")
    spec = scenes.interface_scene(name)
    assert int(g["facet_count"]) == len(spec["facets"])
    s = scenes.build_scene(spec)
    s.render(int(g["spp"]), max_depth=int(g["max_depth"]), seed=77)
    img, _ = s.image()
    a, b = g["image_a"].astype(np.float64), g["image_b"].astype(np.float64)
    d2 = (a - b) ** 2 / 2
    ref = (a + b) / 2
    ratio = ((img - ref) ** 2).sum() / (1.5 * d2.sum())
    z = bias_z(img, a, b, renders=1)
    print(f"{name}: squared difference / predicted noise {ratio:.3f}, bias z {z:.2f}")
    assert 0.7 < ratio < 1.3
    assert abs(z) < 4.5
