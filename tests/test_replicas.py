"""Multi-GPU replicas: sample-range split and the single film reduction.

* The split is a partition of [0, spp) into contiguous ranges (pure host logic).
* The reduction runs as a real 2-rank gloo process group on the CPU: every rank contributes its
  FP64 film sums and receives the total.
* On the GPU, rendering two sample ranges separately and adding their films gives the film of
  one render of all samples (same paths, same generator keys): equal up to the order of the FP64
  atomic additions, i.e. within 1e-12 relative.
"""

import os
import socket

import numpy as np
import pytest

import replicas
import scenes


@pytest.mark.parametrize("spp,world", [(1, 1), (7, 2), (8, 3), (256, 8), (2, 4), (0, 2)])
def test_sample_ranges_partition(spp, world):
    ranges = [replicas.sample_range(spp, r, world) for r in range(world)]
    covered = []
    for first, count in ranges:
        covered.extend(range(first, first + count))
    assert covered == list(range(spp))
    counts = [c for _, c in ranges]
    assert max(counts) - min(counts) <= 1


def test_sample_range_rejects_bad_rank():
    with pytest.raises(ValueError):
        replicas.sample_range(8, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _reduce_worker(rank, world, port, out_dir):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        first, count = replicas.sample_range(10, rank, world)
        # a film whose every sample adds (sample index + 1) to every colour channel, weight 1
        sums = np.full((4, 5, 4), float(sum(range(first + 1, first + count + 1))), np.float64)
        sums[..., 3] = count
        total = replicas.reduce_film(sums, device="cpu")
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), replicas.develop(total))
    finally:
        dist.destroy_process_group()


def test_film_reduction_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_reduce_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    expected = sum(range(1, 11)) / 10.0
    for r in range(2):
        img = np.load(tmp_path / f"rank{r}.npy")
        assert img.shape == (4, 5, 3)
        assert np.allclose(img, expected)


@pytest.mark.gpu
@pytest.mark.parametrize("sample_filter", ["box", "bh"])
def test_split_sample_ranges_reproduce_one_render(gpu_lib, sample_filter):
    import photon_gpu

    scene = scenes.cornell_glossy(32, 32, 8, 8, "bneept")
    with photon_gpu.RenderScene(scene) as whole:
        whole.set_filter(sample_filter)
        whole.render(8, max_bounces=8, seed=9)
        _, ref, _ = whole.film()
    parts = []
    for rank in range(2):
        first, count = replicas.sample_range(8, rank, 2)
        with photon_gpu.RenderScene(scene) as rs:
            rs.set_filter(sample_filter)
            rs.render(count, max_bounces=8, seed=9, first_sample=first)
            parts.append(rs.film()[1])
    total = parts[0] + parts[1]
    assert np.allclose(total, ref, rtol=1e-12, atol=1e-12)
    assert ref.sum() > 0


@pytest.mark.gpu
def test_concurrent_batch_equals_renders_one_by_one(gpu_lib):
    """pgpu_scenes_render with several scenes in flight gives each scene the film it gets from its
    own render (same paths, same generator keys; FP64 atomics only change the addition order)."""
    import photon_gpu

    batch = [scenes.cornell(32, 32, 8, 8, "bneept"), scenes.cornell_glossy(24, 24, 5, 8, "bneept"),
             scenes.ggx_sphere(level=2, width=16, height=16, spp=3, max_bounces=6)]
    alone = []
    for sc in batch:
        with photon_gpu.RenderScene(sc) as rs:
            rs.render(sc.spp, max_bounces=8, seed=5)
            alone.append(rs.film()[1])
    rss = [photon_gpu.RenderScene(sc) for sc in batch]
    try:
        ms = photon_gpu.render_scenes(rss, [sc.spp for sc in batch], max_bounces=8, seed=5, concurrency=3)
        together = [rs.film()[1] for rs in rss]
    finally:
        for rs in rss:
            rs.close()
    assert ms > 0.0
    for a, b in zip(alone, together):
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12)
