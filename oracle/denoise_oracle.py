"""CPU oracle of the learned denoiser (include/ntrace_denoise.h, math_b200/csrc/denoise.cu).

Test infrastructure only: the tests compare the GPU kernels' forward pass, loss and parameter
gradients with this numpy restatement, and check this restatement's own backward pass against
central finite differences.  The denoiser has no counterpart in the reference painter (which only
averages samples), so this oracle restates the network as the C ABI header defines it, not a
reference file.  With bf16=True it rounds to bfloat16 where the GPU does (network inputs, weights,
hidden activations, and the backward products that feed the tensor cores); sums run in float64.
"""

from __future__ import annotations

import numpy as np

HID = 64
TAPS = 9
RADIUS = 4
# cross-bilateral guides (normal, depth, colour): per screen axis the network predicts one
# log-bandwidth o per guide, weighted GUIDE_SCALE x exp(min(o, BANDWIDTH_MAX)) on the tap logits
GUIDES = 3
GUIDE_SCALE = np.array([4.0, 1.0, 0.05])
BANDWIDTH_MAX = 20.0


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    x = np.ascontiguousarray(np.asarray(x, np.float32))
    u = x.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def layout(n: int) -> dict:
    nf = n + 10
    F = nf * (2 * (n - 1) + 1) + 1
    O = (TAPS + GUIDES) * (n - 1)
    return {"n": n, "base_features": nf, "features": F, "outputs": O, "hidden": HID,
            "param_count": HID * F + HID + HID * HID + HID + O * HID + O}


def split(params: np.ndarray, n: int) -> dict:
    L = layout(n)
    F, O = L["features"], L["outputs"]
    out, k = {}, 0
    for name, shape in (("W1", (HID, F)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (O, HID)),
                        ("b3", (O,))):
        size = int(np.prod(shape))
        out[name] = np.asarray(params[k:k + size], np.float64).reshape(shape)
        k += size
    return out


def join(parts: dict) -> np.ndarray:
    return np.concatenate([np.asarray(parts[k], np.float64).reshape(-1) for k in ("W1", "b1", "W2", "b2", "W3", "b3")])


def neighbour_index(screen, a: int, d: int) -> np.ndarray:
    """For every pixel (x0 fastest), the pixel d steps along screen axis a, clamped to the screen."""
    P = int(np.prod(screen))
    idx = np.arange(P)
    stride = int(np.prod(screen[:a]))
    x = (idx // stride) % screen[a]
    y = np.clip(x + d, 0, screen[a] - 1)
    return idx + (y - x) * stride


def base_features(n: int, screen, mean, var, normal, depth) -> np.ndarray:
    """Per-pixel base features (float32): mean (3), standard deviation of the mean (3), normal (n),
    depth / 10, spatial noise estimate (3): sqrt of half the mean squared difference of the mean to
    the 2(n-1) axis neighbours (clamped at the screen's edge)."""
    mean = np.asarray(mean, np.float32).reshape(-1, 3)
    var = np.asarray(var, np.float32).reshape(-1, 3)
    normal = np.asarray(normal, np.float32).reshape(-1, n)
    depth = np.asarray(depth, np.float32).reshape(-1)
    m64 = mean.astype(np.float64)
    sq = np.zeros_like(m64)
    for a in range(n - 1):
        for d in (-1, 1):
            sq += (m64[neighbour_index(screen, a, d)] - m64) ** 2
    spatial = np.sqrt(sq / (4 * (n - 1))).astype(np.float32)
    return np.concatenate([mean, np.sqrt(np.maximum(var, 0)).astype(np.float32), normal,
                           (depth * np.float32(0.1))[:, None], spatial], axis=1)


def guide_distances(base: np.ndarray, n: int, q: np.ndarray) -> np.ndarray:
    """(P, 3) guide distances between every pixel and pixel q of it: squared normal difference,
    squared depth difference, and the non-local-means colour distance (Rousselle, Knaus and Zwicker
    2012): squared mean difference less its noise variance, clamped at 0, over that variance plus
    1e-4 + 0.01 x (average mean)^2, averaged over the channels."""
    bp = np.asarray(base, np.float64)
    bq = bp[q]
    dn = ((bp[:, 6:6 + n] - bq[:, 6:6 + n]) ** 2).sum(axis=1)
    dd = (10.0 * (bp[:, 6 + n] - bq[:, 6 + n])) ** 2
    dm = bp[:, :3] - bq[:, :3]
    v = bp[:, 3:6] ** 2 + bq[:, 3:6] ** 2
    mb = 0.5 * (bp[:, :3] + bq[:, :3])
    dc = (np.maximum(dm ** 2 - v, 0) / (1e-4 + 0.01 * mb ** 2 + v)).sum(axis=1) / 3.0
    return np.stack([dn, dd, dc], axis=1)


def features(n: int, screen, mean, var, normal, depth, spp: int) -> np.ndarray:
    """Network input per pixel: base features (mean, std of the mean, normal, depth / 10, spatial
    noise) at the pixel and at its -1 / +1 neighbours along each screen axis, in that order, then the
    input's noise level 1 / sqrt(spp)."""
    base = base_features(n, screen, mean, var, normal, depth)
    cols = [base]
    for a in range(n - 1):
        cols.append(base[neighbour_index(screen, a, -1)])
        cols.append(base[neighbour_index(screen, a, 1)])
    cols.append(np.full((base.shape[0], 1), 1.0 / np.sqrt(float(spp)), np.float32))
    return np.concatenate(cols, axis=1).astype(np.float32)


def _softmax(z: np.ndarray) -> np.ndarray:
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    return e / e.sum(axis=1, keepdims=True)


def forward(params: np.ndarray, n: int, screen, mean, var, normal, depth, *, spp: int,
            bf16_points: bool = True) -> dict:
    """Denoised image and the intermediate values the backward pass needs."""
    p = split(params, n)
    r = bf16 if bf16_points else (lambda x: np.asarray(x, np.float64))
    X = r(features(n, screen, mean, var, normal, depth, spp)).astype(np.float64)
    if bf16_points:
        W1, W2, W3 = (bf16(p[k].astype(np.float32)).astype(np.float64) for k in ("W1", "W2", "W3"))
    else:
        W1, W2, W3 = p["W1"], p["W2"], p["W3"]
    H1 = np.maximum(X @ W1.T + p["b1"], 0)
    H1 = r(H1.astype(np.float32)).astype(np.float64) if bf16_points else H1
    H2 = np.maximum(H1 @ W2.T + p["b2"], 0)
    H2 = r(H2.astype(np.float32)).astype(np.float64) if bf16_points else H2
    Z = H2 @ W3.T + p["b3"]
    base = base_features(n, screen, mean, var, normal, depth)
    A = n - 1
    ys = [np.asarray(mean, np.float64).reshape(-1, 3)]
    ws, Ds, ss = [], [], []
    for a in range(A):
        o = Z[:, A * TAPS + a * GUIDES:A * TAPS + (a + 1) * GUIDES]
        s = GUIDE_SCALE * np.exp(np.minimum(o, BANDWIDTH_MAX))
        logits = Z[:, a * TAPS:(a + 1) * TAPS].copy()
        D = np.stack([guide_distances(base, n, neighbour_index(screen, a, j - RADIUS)) for j in range(TAPS)], axis=1)
        logits -= (D * s[:, None, :]).sum(axis=2)
        w = _softmax(logits)
        ws.append(w)
        Ds.append(D)
        ss.append(s * (o < BANDWIDTH_MAX))
        y = np.zeros_like(ys[-1])
        for j in range(TAPS):
            y += w[:, j:j + 1] * ys[-1][neighbour_index(screen, a, j - RADIUS)]
        ys.append(y)
    return {"X": X, "W1": W1, "W2": W2, "W3": W3, "H1": H1, "H2": H2, "Z": Z, "ys": ys, "ws": ws, "Ds": Ds,
            "ss": ss, "out": ys[-1]}


def loss_and_grad(params: np.ndarray, n: int, screen, mean, var, normal, depth, target, *, spp: int,
                  bf16_points: bool = True) -> tuple[float, np.ndarray]:
    """Loss sum((out - target)^2) / sum((noisy mean - target)^2) and its gradient (flat, parameter
    order)."""
    f = forward(params, n, screen, mean, var, normal, depth, spp=spp, bf16_points=bf16_points)
    r = (lambda x: bf16(np.asarray(x, np.float32)).astype(np.float64)) if bf16_points else (lambda x: x)
    t = np.asarray(target, np.float64).reshape(-1, 3)
    S = ((f["ys"][0] - t) ** 2).sum()
    diff = f["out"] - t
    loss = float((diff ** 2).sum() / S)
    G = 2 * diff / S
    P = t.shape[0]
    A = n - 1
    dZ = np.zeros((P, (TAPS + GUIDES) * A))
    for a in range(n - 2, -1, -1):
        w = f["ws"][a]
        y_in = f["ys"][a]
        dw = np.zeros((P, TAPS))
        G_in = np.zeros_like(G)
        for j in range(TAPS):
            q = neighbour_index(screen, a, j - RADIUS)
            dw[:, j] = (G * y_in[q]).sum(axis=1)
            np.add.at(G_in, q, w[:, j:j + 1] * G)
        gl = w * (dw - (w * dw).sum(axis=1, keepdims=True))
        dZ[:, a * TAPS:(a + 1) * TAPS] = gl
        # d logit_j / d o_g = -s_g D_g(j) (0 where the log-bandwidth is clamped)
        dZ[:, A * TAPS + a * GUIDES:A * TAPS + (a + 1) * GUIDES] = -(gl[:, :, None] * f["Ds"][a]).sum(axis=1) * f["ss"][a]
        G = G_in
    dZ = r(dZ)
    dH2 = r((dZ @ f["W3"]) * (f["H2"] > 0))
    dH1 = r((dH2 @ f["W2"]) * (f["H1"] > 0))
    grads = {
        "W3": dZ.T @ f["H2"], "b3": dZ.sum(axis=0),
        "W2": dH2.T @ f["H1"], "b2": dH2.sum(axis=0),
        "W1": dH1.T @ f["X"], "b1": dH1.sum(axis=0),
    }
    return loss, join(grads)
