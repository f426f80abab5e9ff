"""Learned denoiser of low-sample renders (include/ntrace_denoise.h), driven from Python.

The network, its training (forward, backward, Adam) and its application run in libntrace's CUDA
kernels (tensor-core GEMMs on tcgen05); this module is the ctypes mirror of that C ABI plus the host
driver: training pairs rendered by the tracer itself (noisy moments + first-hit normal and depth,
and a high-sample target) from seeded variations of a scene (light position, view direction,
albedo), the training loop, and the relative-RMSE measure.  Device arrays are torch CUDA tensors,
used as plumbing (allocation and streams); no torch operator computes the denoiser.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import ntrace
from .ntrace import NtraceError, _check

TAPS = 9
GUIDES = 3  # cross-bilateral guides per screen axis: normal, depth, colour


class Layout(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("base_features", ctypes.c_int), ("features", ctypes.c_int),
                ("features_padded", ctypes.c_int), ("hidden", ctypes.c_int), ("outputs", ctypes.c_int),
                ("outputs_padded", ctypes.c_int), ("param_count", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_bound = False


def _lib() -> ctypes.CDLL:
    global _bound
    lib = ntrace.library()
    if not _bound:
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        sig = {
            "nt_denoiser_create": ([ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)], ctypes.c_int),
            "nt_denoiser_destroy": ([vp], ctypes.c_int),
            "nt_denoiser_get_layout": ([vp, ctypes.POINTER(Layout)], ctypes.c_int),
            "nt_denoiser_get_params": ([vp, vp], ctypes.c_int),
            "nt_denoiser_set_params": ([vp, vp], ctypes.c_int),
            "nt_denoiser_set_input": ([vp, vp, ctypes.c_int, vp, vp, vp, vp, vp], ctypes.c_int),
            "nt_denoiser_apply": ([vp, vp], ctypes.c_int),
            "nt_denoiser_gradient": ([vp, vp, vp, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
            "nt_denoiser_train_step": ([vp, vp, ctypes.c_float, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
            "nt_tc_gemm_bf16": ([vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
            "nt_tc_gemm_wait_selftest": ([vp], ctypes.c_int),
            "nt_tc_gemm_bf16_t": ([vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp], ctypes.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _bound = True
    return lib


def _dev(t) -> int:
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise ValueError("expected a contiguous float32 CUDA tensor")
    return t.data_ptr()


def tc_gemm(a, b):
    """C = A B^T on the tensor cores: A (m x k) and B (n x k) bfloat16 CUDA tensors; C float32."""
    import torch

    if a.dtype != torch.bfloat16 or b.dtype != torch.bfloat16 or not (a.is_cuda and b.is_cuda):
        raise ValueError("expected bfloat16 CUDA tensors")
    a = a.contiguous()
    b = b.contiguous()
    m, k = a.shape
    n, k2 = b.shape
    if k != k2:
        raise ValueError("inner dimensions differ")
    c = torch.empty((m, n), dtype=torch.float32, device=a.device)
    _check(_lib().nt_tc_gemm_bf16(a.data_ptr(), b.data_ptr(), c.data_ptr(), m, n, k,
                                  torch.cuda.current_stream().cuda_stream or None))
    return c


def tc_gemm_t(at, bt, k_per_cta: int = 0):
    """C = At^T Bt on the tensor cores, the weight-gradient form: At (k x m) and Bt (k x n) bfloat16
    CUDA tensors read transposed; the k range split over CTAs of k_per_cta (0: not split); C float32."""
    import torch

    if at.dtype != torch.bfloat16 or bt.dtype != torch.bfloat16 or not (at.is_cuda and bt.is_cuda):
        raise ValueError("expected bfloat16 CUDA tensors")
    at = at.contiguous()
    bt = bt.contiguous()
    k, m = at.shape
    k2, n = bt.shape
    if k != k2:
        raise ValueError("inner dimensions differ")
    c = torch.empty((m, n), dtype=torch.float32, device=at.device)
    _check(_lib().nt_tc_gemm_bf16_t(at.data_ptr(), bt.data_ptr(), c.data_ptr(), m, n, k, k_per_cta,
                                    torch.cuda.current_stream().cuda_stream or None))
    return c


def tc_gemm_wait_selftest() -> int:
    """Runs the GEMM kernel's failure-detection self-test (its completion wait made to run out);
    returns the NT_* status (NT_ETIMEOUT when the kernel detected and reported the timeout)."""
    import torch

    return int(_lib().nt_tc_gemm_wait_selftest(torch.cuda.current_stream().cuda_stream or None))


class Denoiser:
    """A kernel-predicting denoiser for n-dimensional renders (n = 3..6)."""

    def __init__(self, n: int, seed: int = 0):
        self.n = int(n)
        self._lib = _lib()
        h = ctypes.c_void_p()
        _check(self._lib.nt_denoiser_create(self.n, int(seed) & (2 ** 64 - 1), ctypes.byref(h)))
        self._h = h
        lay = Layout()
        _check(self._lib.nt_denoiser_get_layout(self._h, ctypes.byref(lay)))
        self.layout = lay.as_dict()
        self.param_count = int(lay.param_count)
        self.pixels = 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.nt_denoiser_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count, np.float32)
        _check(self._lib.nt_denoiser_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32).reshape(-1))
        if p.size != self.param_count:
            raise ValueError(f"expected {self.param_count} parameters")
        _check(self._lib.nt_denoiser_set_params(self._h, p.ctypes.data))

    def split_params(self, params=None) -> dict:
        """The flat parameter vector as W1, b1, W2, b2, W3, b3."""
        p = self.get_params() if params is None else np.asarray(params, np.float32)
        L = self.layout
        F, H, O = L["features"], L["hidden"], L["outputs"]
        out, k = {}, 0
        for name, shape in (("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))):
            size = int(np.prod(shape))
            out[name] = p[k:k + size].reshape(shape)
            k += size
        return out

    def set_input(self, screen, mean, var, normal, depth, spp: int, stream: int = 0) -> None:
        """The noisy image (device tensors) rendered with spp samples per pixel."""
        scr = np.ascontiguousarray(np.asarray(screen, np.int32))
        if scr.size != self.n - 1:
            raise ValueError("screen needs n - 1 sizes")
        self.pixels = int(np.prod(scr))
        _check(self._lib.nt_denoiser_set_input(self._h, scr.ctypes.data, int(spp), _dev(mean), _dev(var), _dev(normal),
                                               _dev(depth), stream or None))
        self._stream = stream

    def apply(self, out=None):
        import torch

        if out is None:
            out = torch.empty((self.pixels, 3), dtype=torch.float32, device="cuda")
        _check(self._lib.nt_denoiser_apply(self._h, _dev(out)))
        return out

    def gradient(self, target) -> tuple[float, np.ndarray]:
        g = np.zeros(self.param_count, np.float32)
        loss = ctypes.c_double()
        _check(self._lib.nt_denoiser_gradient(self._h, _dev(target), g.ctypes.data, ctypes.byref(loss)))
        return float(loss.value), g

    def train_step(self, target, lr: float = 1e-3) -> float:
        loss = ctypes.c_double()
        _check(self._lib.nt_denoiser_train_step(self._h, _dev(target), float(lr), ctypes.byref(loss)))
        return float(loss.value)

    def save(self, path) -> None:
        np.savez(path, n=self.n, params=self.get_params())

    @classmethod
    def load(cls, path) -> "Denoiser":
        z = np.load(path)
        d = cls(int(z["n"]))
        d.set_params(z["params"])
        return d


# ------------------------------------------------------------------------------------------------
# measures and scene variations


def relative_rmse(a, b) -> float:
    """sqrt(sum (a - b)^2) / sqrt(sum b^2) over pixels and channels (linear RGB)."""
    a = np.asarray(a.detach().cpu() if hasattr(a, "detach") else a, np.float64)
    b = np.asarray(b.detach().cpu() if hasattr(b, "detach") else b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def screen_axes(direction: np.ndarray) -> np.ndarray:
    """Orthonormal screen axes (n-1 rows) perpendicular to a view direction: Gram-Schmidt of
    x_0, x_1, ... against the direction (twice, in double), skipping axes nearly along it, so that a
    view close to -x_(n-1) keeps the default orientation (axis i along +x_i)."""
    d = np.asarray(direction, np.float64)
    n = d.size
    basis = [d / np.linalg.norm(d)]
    for e in np.eye(n):
        v = e.copy()
        for _ in range(2):
            for b in basis:
                v -= np.dot(v, b) * b
        if np.linalg.norm(v) > 0.5:
            basis.append(v / np.linalg.norm(v))
        if len(basis) == n:
            break
    return np.array(basis[1:], np.float32)


def random_variant(n: int, rng: np.random.Generator, screen: int, extent: float = 8.0, max_tilt: float = 0.35,
                   units_per_pixel: float | None = None) -> dict:
    """Seeded light position, albedos in [0.3, 0.9] and a view direction tilted from -x_(n-1).  With
    units_per_pixel the screen is a window of that pixel scale at a seeded place inside the
    extent x ... x extent view (training crops at the scale of a larger evaluation screen)."""
    light = np.concatenate([rng.uniform(-3.0, 3.0, n - 1), rng.uniform(2.0, 4.0, 1)]).astype(np.float32)
    tilt = rng.normal(size=n - 1)
    tilt *= rng.uniform(0.0, max_tilt) / max(np.linalg.norm(tilt), 1e-9)
    d = np.concatenate([tilt, [-1.0]])
    d /= np.linalg.norm(d)
    d = d.astype(np.float32)
    org = -10.0 * d.astype(np.float64)
    upp = extent / screen
    if units_per_pixel is not None:
        upp = float(units_per_pixel)
        half = max(0.0, 0.5 * (extent - screen * upp))
        axes = screen_axes(d).astype(np.float64)
        org = org + (rng.uniform(-half, half, n - 1) @ axes)
    return {
        "light": light,
        "mesh_albedo": float(rng.uniform(0.3, 0.9)),
        "floor_albedo": float(rng.uniform(0.3, 0.9)),
        "dir": d,
        "org": org.astype(np.float32),
        "screen": [screen] * (n - 1),
        "param": upp,
    }


def apply_variant(scene: ntrace.Scene, v: dict, has_floor: bool = True) -> None:
    """Relights and re-aims a scene built from scenes.make_spec (object 0 the mesh, 1 the floor)."""
    scene.clear_lights()
    unit = float(np.linalg.norm(v["light"].astype(np.float64)))
    scene.add_point_light(v["light"], (1.0, 1.0, 1.0), unit)
    a = v["mesh_albedo"]
    scene.set_object_surface(0, (a, a, a), 1.0)
    if has_floor:
        b = v["floor_albedo"]
        scene.set_object_surface(1, (b, b, b), 1.0)
    scene.set_projector(ntrace.PARALLEL, v["org"], v["dir"], screen_axes(v["dir"]), v["param"], v["screen"])
    scene.build()


def render_inputs(scene: ntrace.Scene, spp: int, seed: int, max_depth: int = 5, sample_offset: int = 0,
                  timing: dict | None = None) -> dict:
    """Noisy input of the denoiser: one pass of spp samples per pixel (per-pixel mean and variance of
    the mean) plus the first-hit normal and depth.  timing: filled with the seconds of each part."""
    import torch

    P, n = scene.pixel_count, scene.n
    out = {
        "mean": torch.empty((P, 3), dtype=torch.float32, device="cuda"),
        "var": torch.empty((P, 3), dtype=torch.float32, device="cuda"),
        "normal": torch.empty((P, n), dtype=torch.float32, device="cuda"),
        "depth": torch.empty((P,), dtype=torch.float32, device="cuda"),
    }
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    scene.render_moments(spp, out["mean"].data_ptr(), out["var"].data_ptr(), sample_offset=sample_offset,
                         max_depth=max_depth, seed=seed)
    t1 = time.perf_counter()
    scene.render_aux(out["normal"].data_ptr(), out["depth"].data_ptr())
    if timing is not None:
        torch.cuda.synchronize()
        timing["moments_seconds"] = t1 - t0
        timing["aux_seconds"] = time.perf_counter() - t1
    return out


def render_reference(scene: ntrace.Scene, spp: int, seed: int, max_depth: int = 5):
    """Plain render at spp samples per pixel (stratified), as a CUDA tensor (pixels x 3)."""
    import torch

    scene.clear()
    scene.render(spp, max_depth=max_depth, seed=seed)
    img, _ = scene.image()
    return torch.from_numpy(img).cuda()


def make_pairs(scene: ntrace.Scene, count: int, seed: int, screen: int, spp_in: int, spp_ref: int,
               max_depth: int = 5, has_floor: bool = True, units_per_pixel: float | None = None,
               extent: float = 8.0) -> list[dict]:
    """`count` training pairs from seeded variations of `scene`: spp_in samples per pixel (the noisy
    input with its moments) and spp_ref samples (the target), both stratified."""
    n = scene.n
    rng = np.random.default_rng(seed)
    pairs = []
    for i in range(count):
        v = random_variant(n, rng, screen, extent=extent, units_per_pixel=units_per_pixel)
        apply_variant(scene, v, has_floor)
        x = render_inputs(scene, spp_in, seed=seed * 100003 + 2 * i, max_depth=max_depth)
        x["target"] = render_reference(scene, spp_ref, seed=seed * 100003 + 2 * i + 1, max_depth=max_depth)
        x["screen"] = list(v["screen"])
        x["spp"] = ntrace.effective_spp(n, spp_in)
        pairs.append(x)
    return pairs


def set_pair(den: Denoiser, pair: dict) -> None:
    den.set_input(pair["screen"], pair["mean"], pair["var"], pair["normal"], pair["depth"], pair["spp"])


def train(den: Denoiser, pairs: list[dict], steps: int, lr: float = 1e-3, seed: int = 0, log=None,
          lr_final: float | None = None) -> list[float]:
    """Adam steps over the pairs in a seeded shuffled order; returns the loss of every step.  The
    learning rate is lr throughout, or with lr_final it falls from lr to lr_final along a half cosine."""
    rng = np.random.default_rng(seed)
    losses = []
    order = []
    for s in range(steps):
        if not order:
            order = list(rng.permutation(len(pairs)))
        p = pairs[order.pop()]
        set_pair(den, p)
        rate = lr if lr_final is None else lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * s / max(1, steps)))
        losses.append(den.train_step(p["target"], rate))
        if log and (s % 100 == 0 or s == steps - 1):
            log(f"step {s} loss {losses[-1]:.5f}")
    return losses


def evaluate(den: Denoiser, pairs: list[dict]) -> dict:
    """Relative RMSE of the noisy input, of the untrained-style uniform filter and of the network."""
    import torch

    noisy, den_err = [], []
    for p in pairs:
        set_pair(den, p)
        out = den.apply()
        noisy.append(relative_rmse(p["mean"], p["target"]))
        den_err.append(relative_rmse(out, p["target"]))
    torch.cuda.synchronize()
    return {"noisy": float(np.mean(noisy)), "denoised": float(np.mean(den_err))}


def uniform_filter_params(den: Denoiser) -> np.ndarray:
    """Parameters that make every filter tap weight 1/9 (the method without learning): tap logits 0
    and every guide's log-bandwidth -40 (its weight on the logits below 1e-15)."""
    p = np.zeros(den.param_count, np.float32)
    A = den.n - 1
    p[den.param_count - A * GUIDES:] = -40.0  # the last A x GUIDES biases of the output layer
    return p


def time_call(fn, repeat: int = 1) -> float:
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(repeat):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / repeat


def spp_for_rmse(rmse_at_spp: float, spp: int, target: float) -> float:
    """Samples per pixel at which Monte Carlo error (~ 1/sqrt(spp)) reaches target."""
    return spp * (rmse_at_spp / target) ** 2 if rmse_at_spp > 0 else spp


__all__ = ["Denoiser", "Layout", "tc_gemm", "tc_gemm_t", "relative_rmse", "screen_axes", "random_variant", "apply_variant",
           "render_inputs", "render_reference", "make_pairs", "set_pair", "train", "evaluate",
           "uniform_filter_params", "time_call", "spp_for_rmse", "NtraceError"]
