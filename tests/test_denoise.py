"""Learned denoiser (include/ntrace_denoise.h).

CPU: the oracle's backward pass agrees with central finite differences (float64, no rounding), and
its bfloat16 rounding is round-to-nearest-even.  GPU: the tcgen05 GEMM against a float32 torch
product of the same bfloat16 operands; the network's output, loss and every parameter gradient
against the oracle with the same rounding points; the moments and first-hit inputs against plain
renders; and training on tracer-rendered pairs against the method without learning (every filter
tap 1/9, guides off) on held-out pairs."""

import numpy as np
import pytest

from oracle import denoise_oracle as dor

SPP = 4  # samples per pixel the random inputs claim (the network's noise-level input is 1/2)


def _random_inputs(n, screen, rng):
    P = int(np.prod(screen))
    mean = rng.uniform(0.0, 1.0, (P, 3)).astype(np.float32)
    var = rng.uniform(0.0, 0.05, (P, 3)).astype(np.float32)
    normal = rng.normal(size=(P, n)).astype(np.float32)
    normal /= np.linalg.norm(normal, axis=1, keepdims=True)
    depth = rng.uniform(7.5, 8.5, P).astype(np.float32)
    target = np.clip(mean + rng.normal(0, 0.1, (P, 3)), 0, None).astype(np.float32)
    return mean, var, normal, depth, target


def _random_params(n, rng, scale=0.3):
    L = dor.layout(n)
    p = rng.normal(0, scale, L["param_count"])
    parts = dor.split(p, n)
    parts["W1"] *= 1.0 / np.sqrt(L["features"])
    parts["W2"] *= 1.0 / np.sqrt(dor.HID)
    parts["b1"] = np.abs(parts["b1"]) * 0.1
    parts["b2"] = np.abs(parts["b2"]) * 0.1
    # guide bandwidths of a few units: every guide changes the tap weights without saturating them
    parts["b3"][_bandwidth_columns(n)] += np.tile([-0.75, 0.25, 3.0], n - 1)
    return dor.join(parts)


def _bandwidth_columns(n):
    A = n - 1
    return np.arange(A * dor.TAPS, A * (dor.TAPS + dor.GUIDES))


def _box_params(n):
    """Tap logits 0 and guide bandwidths exp(-40) x scale: the separable 9-tap box filter."""
    L = dor.layout(n)
    parts = dor.split(np.zeros(L["param_count"]), n)
    parts["b3"][_bandwidth_columns(n)] = -40.0
    return dor.join(parts)


def test_gemm_entry_points_validate_their_shapes_before_any_device_work():
    """The GEMM entry points refuse shapes the kernel cannot take (N not a multiple of 16 or above 256;
    for the transposed form M not a multiple of 8) with NT_EINVAL, before touching the device."""
    import ctypes

    from math_b200 import ntrace

    lib = ntrace.library()
    vp = ctypes.c_void_p
    lib.nt_tc_gemm_bf16.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    lib.nt_tc_gemm_bf16_t.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    buf = ctypes.create_string_buffer(64)
    p = ctypes.cast(buf, vp)
    assert lib.nt_tc_gemm_bf16(p, p, p, 16, 8, 16, None) == ntrace.NT_EINVAL
    assert lib.nt_tc_gemm_bf16(p, p, p, 16, 272, 16, None) == ntrace.NT_EINVAL
    assert lib.nt_tc_gemm_bf16(None, p, p, 16, 16, 16, None) == ntrace.NT_EINVAL
    assert lib.nt_tc_gemm_bf16_t(p, p, p, 12, 16, 64, 0, None) == ntrace.NT_EINVAL
    assert lib.nt_tc_gemm_bf16_t(p, p, p, 16, 24, 64, 0, None) == ntrace.NT_EINVAL
    assert lib.nt_tc_gemm_bf16_t(p, p, p, 16, 16, 64, -1, None) == ntrace.NT_EINVAL


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -2.5, 3.0e-39, 1.0 + 2 ** -8 + 2 ** -9], np.float32)
    got = dor.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1); 1 + 1.5 * 2^-8 rounds up
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == np.float32(1.0078125) and got[3] == np.float32(1.0078125)
    assert got[4] == -2.5
    assert got[6] == np.float32(1.0078125)


@pytest.mark.parametrize("n,screen", [(3, (6, 5)), (4, (4, 3, 3))])
def test_oracle_backward_matches_finite_differences(n, screen):
    rng = np.random.default_rng(10 + n)
    mean, var, normal, depth, target = _random_inputs(n, screen, rng)
    params = _random_params(n, rng)
    loss, grad = dor.loss_and_grad(params, n, screen, mean, var, normal, depth, target, spp=SPP, bf16_points=False)
    assert loss > 0
    L = dor.layout(n)
    idx = rng.choice(L["param_count"], 48, replace=False)
    # include the biases and the last layer
    A = n - 1
    bw = L["param_count"] - A * dor.GUIDES  # the first log-bandwidth bias (normal guide of axis 0)
    idx = np.concatenate([idx, [L["param_count"] - 1, L["param_count"] - 10, dor.HID * L["features"] + 3,
                                bw, bw + 1, bw + 2, bw - 1]])
    eps = 1e-6
    for i in idx:
        p1 = params.copy()
        p2 = params.copy()
        p1[i] += eps
        p2[i] -= eps
        l1, _ = dor.loss_and_grad(p1, n, screen, mean, var, normal, depth, target, spp=SPP, bf16_points=False)
        l2, _ = dor.loss_and_grad(p2, n, screen, mean, var, normal, depth, target, spp=SPP, bf16_points=False)
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])


def test_oracle_uniform_filter_is_a_box_blur():
    n, screen = 3, (7, 6)
    rng = np.random.default_rng(3)
    mean, var, normal, depth, _ = _random_inputs(n, screen, rng)
    params = _box_params(n)
    out = dor.forward(params, n, screen, mean, var, normal, depth, spp=SPP, bf16_points=False)["out"]
    # interior pixel: mean of the 9 x 9 neighbourhood (separable, clamped at the border)
    x0, x1 = 3, 3
    img = mean.reshape(screen[1], screen[0], 3).astype(np.float64)
    cols = np.clip(np.arange(x0 - 4, x0 + 5), 0, screen[0] - 1)
    rows = np.clip(np.arange(x1 - 4, x1 + 5), 0, screen[1] - 1)
    expect = img[np.ix_(rows, cols)].reshape(-1, 3).mean(axis=0)
    np.testing.assert_allclose(out[x1 * screen[0] + x0], expect, rtol=1e-12)


def test_oracle_input_features_layout():
    """Input row: (n + 10) base features at the pixel and its 2(n-1) axis neighbours, then the noise
    level 1/sqrt(spp); the spatial noise estimate is 0 on a constant image and close to the noise's
    standard deviation on independent noise."""
    n, screen = 4, (9, 8, 7)
    P = int(np.prod(screen))
    rng = np.random.default_rng(21)
    normal = np.tile([0.0, 0.0, 0.0, 1.0], (P, 1)).astype(np.float32)
    depth = np.full(P, 8.0, np.float32)
    var = np.zeros((P, 3), np.float32)
    flat = np.full((P, 3), 0.4, np.float32)
    X = dor.features(n, screen, flat, var, normal, depth, 9)
    L = dor.layout(n)
    nf = n + 10
    assert X.shape == (P, L["features"]) and L["features"] == nf * (2 * (n - 1) + 1) + 1
    np.testing.assert_array_equal(X[:, -1], np.float32(1.0 / 3.0))
    np.testing.assert_array_equal(X[:, 7 + n:10 + n], 0.0)  # spatial noise of a constant image
    # the -1 neighbour along axis 1 of pixel (x0, x1, x2) = (4, 3, 2) is (4, 2, 2)
    mean = rng.uniform(0, 1, (P, 3)).astype(np.float32)
    X = dor.features(n, screen, mean, var, normal, depth, 1)
    p = 4 + 9 * (3 + 8 * 2)
    q = 4 + 9 * (2 + 8 * 2)
    np.testing.assert_array_equal(X[p, 3 * nf:3 * nf + 3], mean[q])
    sigma = 0.05
    noisy = (0.5 + rng.normal(0, sigma, (P, 3))).astype(np.float32)
    spatial = dor.base_features(n, screen, noisy, var, normal, depth)[:, 7 + n:10 + n]
    interior = spatial.reshape(screen[2], screen[1], screen[0], 3)[1:-1, 1:-1, 1:-1]
    assert abs(float(np.sqrt((interior.astype(np.float64) ** 2).mean())) - sigma) < 0.15 * sigma


def test_oracle_normal_guide_keeps_edges():
    """Two half-screens of different normal: with tap logits 0 and the normal guide at 64 per unit of
    squared normal difference (log-bandwidth ln 16 over its base 4), each half is averaged over
    itself only."""
    n, screen = 3, (12, 5)
    P = screen[0] * screen[1]
    x0 = np.arange(P) % screen[0]
    left = x0 < 6
    rng = np.random.default_rng(8)
    mean = np.where(left[:, None], 0.2, 0.7) + rng.uniform(-0.05, 0.05, (P, 3))
    var = np.full((P, 3), 1e-2, np.float32)
    normal = np.where(left[:, None], [0.0, 0.0, 1.0], [0.6, 0.0, 0.8]).astype(np.float32)
    depth = np.full(P, 8.0, np.float32)
    params = _box_params(n)
    parts = dor.split(params.copy(), n)
    parts["b3"][_bandwidth_columns(n)[0::dor.GUIDES]] = np.log(16.0)  # normal guide on, at 64
    out = dor.forward(dor.join(parts), n, screen, mean, var, normal, depth, spp=SPP, bf16_points=False)["out"]
    box = dor.forward(params, n, screen, mean, var, normal, depth, spp=SPP, bf16_points=False)["out"]
    # |n_l - n_r|^2 = 0.4: every tap across the edge is weighted exp(-25.6) against the same side
    for side, level in ((left, 0.2), (~left, 0.7)):
        assert np.abs(out[side] - level).max() < 0.05
    assert np.abs(box[x0 == 5] - 0.2).max() > 0.1  # the box filter mixes the halves at the edge


# ------------------------------------------------------------------------------------------------
# GPU


def _torch():
    import torch

    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k", [(1, 16, 16), (127, 64, 64), (300, 48, 112), (1000, 144, 80), (129, 256, 144),
                                   (4096, 64, 64)])
def test_tc_gemm_matches_torch(require_gpu, m, n, k):
    torch = _torch()
    from math_b200.denoise import tc_gemm

    g = torch.Generator(device="cpu").manual_seed(m * 7 + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(n, k, generator=g).to(torch.bfloat16).cuda()
    c = tc_gemm(a, b)
    ref = a.float() @ b.float().T
    err = (c - ref).abs().max().item()
    assert err <= 1e-3 * max(1.0, ref.abs().max().item()), err


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k,kpc", [(8, 16, 16, 0), (64, 64, 4096, 1024), (144, 64, 3000, 512),
                                       (136, 48, 200, 0), (128, 256, 130, 64)])
def test_tc_gemm_transposed_split_matches_torch(require_gpu, m, n, k, kpc):
    """The weight-gradient form: both operands read MN-major (transposed row-major matrices), ragged
    k, and the k range split over CTAs with FP32 atomics."""
    torch = _torch()
    from math_b200.denoise import tc_gemm_t

    g = torch.Generator(device="cpu").manual_seed(m + 3 * n + k)
    at = torch.randn(k, m, generator=g).to(torch.bfloat16).cuda()
    bt = torch.randn(k, n, generator=g).to(torch.bfloat16).cuda()
    c = tc_gemm_t(at, bt, kpc)
    ref = at.float().T @ bt.float()
    err = (c - ref).abs().max().item()
    assert err <= 1e-3 * max(1.0, ref.abs().max().item()), err


@pytest.mark.gpu
def test_tc_gemm_wait_runs_out_and_reports(require_gpu):
    """Failure detection without a fault: the GEMM kernel with its tensor-core instructions withheld
    (nothing ever arrives on its barrier) gives up its bounded wait, frees its tensor memory and reports
    NT_ETIMEOUT; the context stays usable (an ordinary GEMM right after is correct)."""
    torch = _torch()
    from math_b200 import ntrace
    from math_b200.denoise import tc_gemm, tc_gemm_wait_selftest

    assert tc_gemm_wait_selftest() == ntrace.NT_ETIMEOUT
    assert b"completion wait ran out" in ntrace.library().nt_last_error_message()
    g = torch.Generator(device="cpu").manual_seed(5)
    a = torch.randn(256, 64, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(32, 64, generator=g).to(torch.bfloat16).cuda()
    c = tc_gemm(a, b)
    ref = a.float() @ b.float().T
    assert (c - ref).abs().max().item() <= 1e-3 * ref.abs().max().item()


def _gpu_inputs(n, screen, seed):
    torch = _torch()
    mean, var, normal, depth, target = _random_inputs(n, screen, np.random.default_rng(seed))
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
         dict(mean=mean, var=var, normal=normal, depth=depth, target=target).items()}
    return (mean, var, normal, depth, target), t


@pytest.mark.gpu
@pytest.mark.parametrize("n,screen", [(3, (33, 20)), (4, (9, 8, 7)), (5, (6, 5, 4, 4))])
def test_forward_loss_and_gradients_match_oracle(require_gpu, n, screen):
    from math_b200.denoise import Denoiser

    (mean, var, normal, depth, target), t = _gpu_inputs(n, screen, 100 + n)
    den = Denoiser(n, seed=5)
    params = _random_params(n, np.random.default_rng(n)).astype(np.float32)
    den.set_params(params)
    den.set_input(screen, t["mean"], t["var"], t["normal"], t["depth"], SPP)
    out = den.apply().cpu().numpy()
    ref = dor.forward(params, n, screen, mean, var, normal, depth, spp=SPP, bf16_points=True)
    rel = np.linalg.norm(out - ref["out"]) / np.linalg.norm(ref["out"])
    assert rel < 2e-3, rel
    loss, grad = den.gradient(t["target"])
    loss_o, grad_o = dor.loss_and_grad(params, n, screen, mean, var, normal, depth, target, spp=SPP, bf16_points=True)
    assert abs(loss - loss_o) <= 2e-3 * loss_o, (loss, loss_o)
    gp = dor.split(grad, n)
    go = dor.split(grad_o, n)
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        e = np.linalg.norm(gp[name] - go[name]) / max(np.linalg.norm(go[name]), 1e-30)
        assert e < 2e-2, (name, e)


@pytest.fixture(scope="module")
def n3_pairs():
    from math_b200 import denoise, scenes

    v, f = scenes.icosphere(3)
    spec = scenes.make_spec(3, v, f, screen=32, spp=4, max_depth=5, seed=0)
    scene = scenes.build_scene(spec)
    pairs = denoise.make_pairs(scene, 30, seed=7, screen=32, spp_in=4, spp_ref=1024)
    return scene, pairs


@pytest.mark.gpu
def test_moments_and_first_hit_inputs(require_gpu):
    torch = _torch()
    from math_b200 import denoise, scenes

    v, f = scenes.icosphere(2)
    spec = scenes.make_spec(3, v, f, screen=24, spp=4, max_depth=3, seed=0)
    scene = scenes.build_scene(spec)
    x = denoise.render_inputs(scene, 4, seed=11, max_depth=3)
    # the same pass through the ordinary render (same samples, summed per pixel) gives the same mean
    scene.clear()
    scene.render(4, max_depth=3, seed=11)
    plain, spp = scene.image()
    assert spp == 4
    np.testing.assert_allclose(x["mean"].cpu().numpy(), plain, rtol=1e-5, atol=1e-6)
    var = x["var"].cpu().numpy()
    assert (var >= 0).all() and var.max() > 0
    normal = x["normal"].cpu().numpy()
    depth = x["depth"].cpu().numpy()
    hit = depth > 0
    assert hit.all()  # the floor fills the screen
    np.testing.assert_allclose(np.linalg.norm(normal[hit], axis=1), 1.0, rtol=1e-5)
    # every normal faces the camera (which looks along -x2)
    assert (normal[:, 2] >= 0).all()
    # the pixel under the sphere's top sees the sphere at distance 10 - 1 (camera at x2 = 10)
    centre = 12 * 24 + 12
    assert abs(depth[centre] - 9.0) < 0.05, depth[centre]
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_training_beats_the_uniform_filter(require_gpu, n3_pairs):
    from math_b200 import denoise

    scene, pairs = n3_pairs
    train, held = pairs[:24], pairs[24:]
    den = denoise.Denoiser(3, seed=1)
    den.set_params(denoise.uniform_filter_params(den))
    uniform = denoise.evaluate(den, held)
    den2 = denoise.Denoiser(3, seed=1)
    losses = denoise.train(den2, train, steps=400, lr=2e-3, seed=3)
    assert np.mean(losses[-50:]) < np.mean(losses[:50])
    trained = denoise.evaluate(den2, held)
    assert trained["denoised"] < trained["noisy"]
    assert trained["denoised"] < 0.9 * uniform["denoised"], (trained, uniform)
