"""Launch-shape autotuner (pgpu_scene_autotune / phGpuAutotune).

The reference has no counterpart: its EqualSamplingRenderer fixes its scheduler and tiles up front
(Engine/Source/Core/Renderer/Sampling/EqualSamplingRenderer.cpp:45-60). Launch shapes change how
paths are scheduled onto the GPU, never which paths are traced: every path draws its numbers from
a generator keyed by its own index, so an image rendered with tuned shapes is the default image up
to the order of FP64 film additions (and, where the BVH leaf size changes, the traversal's
near-ties between coincident triangles).
"""

import numpy as np
import pytest

import scenes


def _rel_mse(x, ref, eps=1e-2):
    return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + eps)))


@pytest.mark.gpu
def test_autotune_picks_shapes_caches_them_and_keeps_the_image(gpu_lib, tmp_path):
    import photon_gpu

    scene = scenes.ggx_sphere(level=5, width=128, height=128, spp=64, max_bounces=10)
    cache = str(tmp_path / "tuning.txt")
    with photon_gpu.RenderScene(scene) as rs:
        assert rs.launch() == {"capacity": 1 << 21, "refill": 8, "blocks_per_sm": 8, "leaf_tris": 3}
        rs.render(64, max_bounces=10, seed=9)
        default_img = rs.film(with_sums=False)[0]
        tuned = rs.autotune(64, max_bounces=10, rebuild=True, cache_path=cache)
        print(f"autotune: {tuned}")
        assert tuned["capacity"] in (1 << 19, 1 << 20, 1 << 21, 1 << 22)
        assert tuned["refill"] in (4, 8, 12, 16) and tuned["blocks_per_sm"] in (4, 8, 16)
        assert tuned["leaf_tris"] in (1, 2, 3)
        assert tuned["ms_tuned"] <= tuned["ms_default"] and tuned["trials"] > 0 and not tuned["from_cache"]
        assert rs.launch() == {k: tuned[k] for k in ("capacity", "refill", "blocks_per_sm", "leaf_tris")}
        rs.clear()
        rs.render(64, max_bounces=10, seed=9)
        tuned_img = rs.film(with_sums=False)[0]
        assert _rel_mse(tuned_img, default_img) < 1e-8
        # the same scene again: the cache answers without calibrating
        again = rs.autotune(64, max_bounces=10, rebuild=True, cache_path=cache)
        assert again["from_cache"] and again["trials"] == 0
        assert {k: again[k] for k in ("capacity", "refill", "blocks_per_sm", "leaf_tris")} == \
               {k: tuned[k] for k in ("capacity", "refill", "blocks_per_sm", "leaf_tris")}
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith("tris=")


@pytest.mark.gpu
def test_launch_shapes_rebuild_and_validation(gpu_lib):
    """Each leaf size renders the same image (the hit a ray finds does not depend on the tree);
    shapes outside their ranges are rejected."""
    import photon_gpu

    scene = scenes.cornell(64, 64, 32, 8, "bneept")
    with photon_gpu.RenderScene(scene) as rs:
        images = []
        for leaf, capacity, refill, blocks in ((3, 1 << 21, 8, 8), (1, 1 << 19, 4, 16), (2, 1 << 20, 16, 4)):
            rs.set_launch(capacity=capacity, refill=refill, blocks_per_sm=blocks, leaf_tris=leaf)
            assert rs.launch()["leaf_tris"] == leaf
            rs.clear()
            rs.render(32, max_bounces=8, seed=4)
            images.append(rs.film(with_sums=False)[0])
        for img in images[1:]:
            assert _rel_mse(img, images[0]) < 1e-8
        for bad in ({"capacity": 10}, {"refill": 0}, {"refill": 33}, {"blocks_per_sm": 0}, {"leaf_tris": 4}):
            with pytest.raises(photon_gpu.PhotonGpuError):
                rs.set_launch(**bad)


@pytest.mark.gpu
def test_photon_api_autotune(gpu_lib, tmp_path):
    """phGpuAutotune tunes the updated scene of a Photon engine for its session settings."""
    import photon_gpu

    scene = scenes.cornell(64, 64, 16, 8, "bneept")
    p2 = tmp_path / "scene.p2"
    p2.write_text(scenes.to_sdl(scene))
    with photon_gpu.PhotonEngine() as eng:
        eng.set_working_directory(str(tmp_path))
        assert eng.load_file(str(p2)), eng.errors()
        eng.set_max_bounces(8)
        eng.update()
        t = eng.autotune(rebuild=False)
        assert t["trials"] > 0 and t["leaf_tris"] == 3
        eng.render()
        assert eng.info()["paths"] == 64 * 64 * 16
