"""nt_render_noalloc: rendering for callers that cannot allocate device memory (marked gpu).

Applications that own all device memory through their own allocator or a budget fixed at start-up,
and frame loops where an allocation is not allowed, render through this entry point: its wavefront
working memory is a fixed array inside the library and the image sums go to the caller's buffer.
The test calls it through the C ABI twice in a row (two passes, the second continuing the sample
sequence) and compares the result with the ordinary nt_render of the same two passes, within the
relative-RMSE tolerance the GPU radiance tests use (1e-4).  This file is collected last so that a run
stopping at its first failure has run every other test before it.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOLERANCE = 1e-4
SCRATCH_BYTES = 64 << 20  # NT_NOALLOC_SCRATCH_BYTES


def _bind():
    from math_b200 import ntrace

    lib = ntrace.library()
    fn = lib.nt_render_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(ntrace.RenderOpts), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                   ctypes.POINTER(ntrace.Stats)]
    fn.restype = ctypes.c_int
    return ntrace, fn


def _opts(ntrace, spp, depth, seed, pool_paths=0):
    return ntrace.RenderOpts(spp, depth, seed, 1, 0, pool_paths, 0, None)


def _rrmse(a, b):
    return float(np.sqrt(((a - b) ** 2).sum()) / np.sqrt((b ** 2).sum()))


@pytest.mark.parametrize("name", ["n3_small", "n4_small"])
def test_noalloc_render_matches_render(require_gpu, name):
    import torch

    from math_b200 import scenes

    ntrace, render_noalloc = _bind()
    spec = scenes.config(name)
    scene = scenes.build_scene(spec)
    spp, depth, seed = spec["spp"], spec["max_depth"], 11
    spp_eff = ntrace.effective_spp(spec["n"], spp)

    # the ordinary entry point: two passes
    scene.render(spp, max_depth=depth, seed=seed)
    scene.render(spp, max_depth=depth, seed=seed)
    expect, done = scene.image()
    assert done == 2 * spp_eff

    # the no-alloc entry point: two calls in a row into a caller-owned accumulator
    acc = torch.zeros((scene.pixel_count, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = ntrace.Stats()
    # the first call on the device may load the library's module that holds the fixed array (lazy module
    # loading), which reserves the array then and nothing beyond it
    free_first = torch.cuda.mem_get_info()[0]
    code = render_noalloc(scene._h, ctypes.byref(_opts(ntrace, spp, depth, seed)), acc.data_ptr(), 0, None,
                          ctypes.byref(st))
    assert code == ntrace.NT_OK, ntrace.library().nt_last_error_message()
    assert free_first - torch.cuda.mem_get_info()[0] <= SCRATCH_BYTES + (8 << 20)
    assert st.paths == scene.pixel_count * spp_eff and st.error_bits == 0 and st.iterations > 0
    free_before = torch.cuda.mem_get_info()[0]
    code = render_noalloc(scene._h, ctypes.byref(_opts(ntrace, spp, depth, seed)), acc.data_ptr(), spp_eff, None,
                          ctypes.byref(st))
    assert code == ntrace.NT_OK, ntrace.library().nt_last_error_message()
    assert st.paths == scene.pixel_count * spp_eff and st.error_bits == 0 and st.iterations > 0
    assert torch.cuda.mem_get_info()[0] == free_before
    got = (acc / (2 * spp_eff)).cpu().numpy().astype(np.float32)
    assert _rrmse(got, expect) < TOLERANCE

    # a pool larger than the fixed array is refused with a clear error
    code = render_noalloc(scene._h, ctypes.byref(_opts(ntrace, spp, depth, seed, pool_paths=1 << 40)),
                          acc.data_ptr(), 0, None, ctypes.byref(st))
    assert code == ntrace.NT_EINVAL
    assert b"no-alloc scratch capacity" in ntrace.library().nt_last_error_message()
