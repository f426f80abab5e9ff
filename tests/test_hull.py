"""Exact convex hull (nt_convex_hull): the boundary facets of the measured scenes' point sets.

Points in general position have one hull, whatever the algorithm: the facet set must equal Qhull's
(scipy) on seeded sphere points in 3..6 dimensions, interior points never appear, duplicate points
are dropped, and a point set that spans fewer dimensions is rejected."""

import numpy as np
import pytest

from scipy.spatial import ConvexHull


def _facet_set(f):
    return set(tuple(sorted(int(i) for i in x)) for x in f)


@pytest.mark.parametrize("n,count", [(3, 3000), (4, 1500), (5, 400), (6, 120)])
def test_hull_equals_qhull_on_sphere_points(n, count):
    from math_b200 import ntrace, scenes

    pts = scenes.sphere_points(n, count, seed=7 + n)
    mine = ntrace.convex_hull(pts)
    ref = ConvexHull(pts.astype(np.float64)).simplices
    assert mine.shape[1] == n
    assert _facet_set(mine) == _facet_set(ref)


def test_interior_and_duplicate_points_are_not_vertices():
    from math_b200 import ntrace, scenes

    rng = np.random.default_rng(1)
    shell = scenes.sphere_points(4, 500, seed=2)
    inner = (rng.standard_normal((300, 4)) * 0.05).astype(np.float32)
    pts = np.concatenate([shell, inner, shell[:50]])
    f = ntrace.convex_hull(pts)
    used = set(np.unique(f))
    assert used.isdisjoint(range(500, 800))
    # the duplicated shell points appear once (either copy), and the hull is the shell's
    ref = _facet_set(ConvexHull(shell.astype(np.float64)).simplices)
    canon = np.where(f >= 800, f - 800, f)
    assert _facet_set(canon) == ref


def test_flat_point_set_is_rejected():
    from math_b200 import ntrace

    rng = np.random.default_rng(3)
    pts = np.zeros((100, 4), np.float32)
    pts[:, :3] = rng.standard_normal((100, 3))
    with pytest.raises(ntrace.NtraceError):
        ntrace.convex_hull(pts)
