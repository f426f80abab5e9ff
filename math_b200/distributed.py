"""Several GPUs on one frame: sample-range sharding.

Pixels and samples of a frame are independent and the scene is read-only, so every rank renders the
whole screen with its own range of sample indices (the path id of sample s of pixel p is
s * pixel_count + p, so disjoint ranges trace disjoint paths) and the per-pixel sums are combined once,
after rendering, with one all-reduce.  There is no exchange inside a frame.
"""

from __future__ import annotations

import numpy as np


def sample_offset(rank: int, passes_before: int, spp_effective: int, world: int) -> int:
    """First sample index of a rank's pass: ranks interleave whole passes (pass k of rank r covers
    samples [(k * world + r) * spp, (k * world + r + 1) * spp))."""
    return (passes_before * world + rank) * spp_effective


def combine(mean_rgb: np.ndarray, samples: int, group=None) -> tuple[np.ndarray, int]:
    """All-reduce of the ranks' per-pixel sums (mean x samples) and sample counts over the default
    process group (or ``group``); returns the combined mean image and the total samples per pixel."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    device = "cuda" if backend == "nccl" else "cpu"
    sums = torch.from_numpy(mean_rgb.astype(np.float64) * samples).to(device)
    count = torch.tensor([float(samples)], dtype=torch.float64, device=device)
    dist.all_reduce(sums, group=group)
    dist.all_reduce(count, group=group)
    total = int(count.item())
    return (sums / max(total, 1)).cpu().numpy().astype(np.float32), total
