"""Graph-captured wavefront, batches of scenes and the autotuner (include/ntrace.h).

The wavefront keeps its queue sizes on the device, so its iterations can be captured as a CUDA graph
(the default), enqueued one by one (timing), or interleaved with other scenes' passes in one graph
(nt_render_batch).  Every form traces the same paths: images agree to FP64 summation-order rounding."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rrmse(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def _scene(name):
    from math_b200 import scenes

    spec = scenes.config(name)
    return spec, scenes.build_scene(spec)


def test_graph_and_direct_iterations_trace_the_same_paths(require_gpu):
    spec, s = _scene("n4_small")
    st_g = s.render(spec["spp"], max_depth=spec["max_depth"], seed=4)
    img_g, _ = s.image()
    s.clear()
    st_d = s.render(spec["spp"], max_depth=spec["max_depth"], seed=4, timing=True)
    img_d, _ = s.image()
    assert rrmse(img_g, img_d) < 1e-12
    for k in ("rays", "shadow_rays", "facet_tests", "box_steps", "retests", "iterations"):
        assert st_g[k] == st_d[k], k
    assert st_g["iterations"] > 0 and st_d["extend_ms"] > 0
    # every graph-iteration count gives the same image
    for it in (1, 2, 8):
        s.clear()
        s.render(spec["spp"], max_depth=spec["max_depth"], seed=4, graph_iterations=it, pool_paths=1000)
        img, _ = s.image()
        assert rrmse(img, img_d) < 1e-12, it


@pytest.mark.parametrize("name", ["n3_small", "n4_small", "n5_small", "n6_small"])
def test_walk_chunks_trace_the_same_paths(require_gpu, name):
    """The walk kernels' variant (records read directly, or staged in chunks of 32, 64 or 128 pooled
    facet tests per warp) and small-leaf threshold (leaves tested lane by lane below it, pooled across
    the warp above it) are tuning choices only: every combination makes the same decisions (same work
    counters, same image)."""
    spec, s = _scene(name)
    ref = None
    for chunk, small in ((1, 2), (32, 2), (64, 2), (128, 2), (1, -1), (1, 4), (32, 8)):
        s.clear()
        st = s.render(spec["spp"], max_depth=spec["max_depth"], seed=6, walk_chunk=chunk, walk_small_leaf=small)
        img, _ = s.image()
        assert st["error_bits"] == 0
        if ref is None:
            ref = (st, img)
            continue
        for k in ("rays", "shadow_rays", "facet_tests", "box_steps", "retests", "shadow_facet_tests",
                  "shadow_box_steps"):
            assert st[k] == ref[0][k], (chunk, small, k)
        assert rrmse(img, ref[1]) < 1e-12, (chunk, small)


@pytest.mark.parametrize("name", ["n3_small", "n4_small", "n5_small"])
def test_records_through_index_lists_trace_the_same_paths(require_gpu, name):
    """Without the leaf-ordered record copy (nt_build_opts.leaf_records = -1, what a mesh gets when the
    copy would not fit a quarter of the free memory) the walk reads a leaf's records through its index
    list: same decisions (work counters), same image, for the direct and the staged walk variants."""
    from math_b200 import scenes

    spec = scenes.config(name)
    a = scenes.build_scene(spec)
    b = scenes.build_scene(spec, leaf_records=-1)
    assert a.mesh_info(0)["device_bytes"] > b.mesh_info(0)["device_bytes"]
    for chunk in (1, 32):
        imgs, sts = [], []
        for s in (a, b):
            s.clear()
            sts.append(s.render(spec["spp"], max_depth=spec["max_depth"], seed=8, walk_chunk=chunk))
            imgs.append(s.image()[0])
        for k in ("rays", "shadow_rays", "facet_tests", "box_steps", "retests", "shadow_facet_tests",
                  "shadow_box_steps", "descent_levels"):
            assert sts[0][k] == sts[1][k], (chunk, k)
        assert rrmse(imgs[1], imgs[0]) < 1e-12, chunk


def test_walk_chunk_is_validated(require_gpu):
    from math_b200 import ntrace

    spec, s = _scene("n3_small")
    with pytest.raises(ntrace.NtraceError) as e:
        s.render(spec["spp"], walk_chunk=48)
    assert e.value.code == ntrace.NT_EINVAL


def test_batch_of_mixed_dimensions_matches_single_renders(require_gpu):
    from math_b200 import ntrace

    names = ["n3_small", "n4_small", "n5_small", "n6_small"]
    built = [_scene(nm) for nm in names]
    singles = []
    for spec, s in built:
        s.render(spec["spp"], max_depth=spec["max_depth"], seed=9)
        singles.append(s.image()[0])
        s.clear()
    opts = [dict(samples_per_pixel=spec["spp"], max_depth=spec["max_depth"], seed=9) for spec, _ in built]
    stats = ntrace.render_batch([s for _, s in built], opts)
    for (spec, s), single, st in zip(built, singles, stats):
        img, spp = s.image()
        assert spp == ntrace.effective_spp(spec["n"], spec["spp"])
        assert st["error_bits"] == 0 and st["paths"] == s.pixel_count * spp
        assert rrmse(img, single) < 1e-12


def test_batch_rejects_repeated_scene(require_gpu):
    from math_b200 import ntrace

    spec, s = _scene("n3_small")
    with pytest.raises(ntrace.NtraceError):
        ntrace.render_batch([s, s], [dict(samples_per_pixel=1), dict(samples_per_pixel=1)])


def test_autotune_picks_a_candidate_and_clears(require_gpu):
    spec, s = _scene("n4_small")
    tuned, ms = s.autotune(spec["spp"], max_depth=spec["max_depth"])
    assert tuned["graph_iterations"] in (2, 4, 8, 16)
    assert tuned["walk_chunk"] in (1, 32, 64, 128)
    assert tuned["pool_paths"] >= 256 and ms > 0
    img, spp = s.image()
    assert spp == 0 and not img.any()
    s.render(spec["spp"], max_depth=spec["max_depth"], seed=1, **tuned)
    assert s.image()[1] > 0
