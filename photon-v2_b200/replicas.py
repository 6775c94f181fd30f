"""Multi-GPU rendering by sample-range replicas: one process per GPU, one film reduction.

Paths are independent, so a render of S samples per pixel splits into disjoint, contiguous
sample ranges, one per rank. Every rank renders its range on its own GPU with the same seed. The
path generator keys each path by its global index (sample index x pixels + pixel), so the union
of the ranges is exactly the set of paths one GPU would trace for all S samples. The FP64 film
sums (filter-weighted R, G, B and the weight W per pixel) then meet in a single all-reduce, and
the developed image is RGB / W.

This is the multi-device analogue of the reference's split of one render across worker threads,
each with its own film merged into the main film (EqualSamplingRenderer::doRender,
Engine/Engine/Source/Core/Renderer/Sampling/EqualSamplingRenderer.cpp:123-190). There is no
exchange on the data path: the only collective is the final reduction of W x H x 4 doubles.
"""

from __future__ import annotations

from typing import Tuple

import numpy as np


def sample_range(spp: int, rank: int, world: int) -> Tuple[int, int]:
    """(first sample, sample count) of `rank` when `spp` samples are split over `world` ranks.

    Ranges are contiguous, disjoint and cover [0, spp); counts differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    if spp < 0:
        raise ValueError("negative sample count")
    base, extra = divmod(spp, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def reduce_film(sums: np.ndarray, group=None, device: str = "cpu") -> np.ndarray:
    """Sums the ranks' FP64 film sums (all-reduce); every rank receives the total.

    `device` is where the reduction runs: "cpu" for a gloo group, "cuda" for NCCL."""
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.ascontiguousarray(sums, np.float64)).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def develop(sums: np.ndarray) -> np.ndarray:
    """Develop of FP64 (R, G, B, W) sums [..., 4]: RGB / W, 0 where W is 0
    (HdrRgbFilm::developRegion, Engine/Engine/Source/Core/Filmic/HdrRgbFilm.cpp:167-205)."""
    if sums.shape[-1] != 4:
        raise ValueError("film sums must be [..., 4] (R, G, B, W)")
    w = sums[..., 3:4]
    rcp = np.divide(1.0, w, out=np.zeros_like(w), where=w != 0)
    return (sums[..., :3] * rcp).astype(np.float32)


def render_replicated(scene, spp: int, rank: int, world: int, max_bounces: int = 10000,
                      estimator: int = 0, seed: int = 42, group=None, reduce_device: str = "cuda"):
    """Renders this rank's sample range of `scene` (a ``scenes.Scene``) on the current GPU and
    returns the developed image of all ranks' samples. Every rank must call it (collective)."""
    import photon_gpu

    first, count = sample_range(spp, rank, world)
    with photon_gpu.RenderScene(scene) as rs:
        if count:
            rs.render(count, max_bounces=max_bounces, estimator=estimator, seed=seed, first_sample=first)
        _, sums, _ = rs.film()
    total = reduce_film(sums, group=group, device=reduce_device)
    return develop(total)
