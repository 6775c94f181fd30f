"""Many scenes rendered as one wavefront (pgpu_scenes_render_wavefront).

One path pool serves all scenes and every kernel is launched once per iteration for all of them:
queue entries carry their scene, and each path takes its scene's camera, tree, materials, lights
and film. The reference renders scene after scene, one EqualSamplingRenderer each
(Engine/Source/Core/Renderer/Sampling/EqualSamplingRenderer.cpp:119-203). Every path draws the
numbers of its index within its own scene, so each scene's film must equal the film of its own
render with the same seed up to the order of FP64 additions (relMSE below 1e-12, weights equal).
"""

import dataclasses

import numpy as np
import pytest

import scenes


def _scenes():
    return [
        scenes.cornell(64, 48, 24, 8, "bneept"),
        scenes.ggx_sphere(level=4, width=96, height=64, spp=8, max_bounces=10),
        dataclasses.replace(scenes.batch_scene(0), width=80, height=80, spp=12),
        scenes.cornell_glossy(40, 40, 16, 8, "bneept"),
        dataclasses.replace(scenes.batch_scene(3), width=72, height=56, spp=5),
    ]


def _rel(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


@pytest.mark.gpu
@pytest.mark.parametrize("estimator", ["bneept", "bvpt"])
def test_wavefront_equals_scene_by_scene(gpu_lib, estimator):
    import photon_gpu

    est = {"bneept": photon_gpu.BNEEPT, "bvpt": photon_gpu.BVPT}[estimator]
    sc = _scenes()
    rss = [photon_gpu.RenderScene(s) for s in sc]
    try:
        solo = []
        for s, rs in zip(sc, rss):
            rs.render(s.spp, max_bounces=10, estimator=est, seed=77)
            solo.append(rs.film())
            rs.clear()
        ms = photon_gpu.render_scenes_wavefront(rss, [s.spp for s in sc], max_bounces=10, estimator=est, seed=77)
        assert ms > 0.0
        for s, rs, (rgb0, sums0, spp0) in zip(sc, rss, solo):
            rgb, sums, spp = rs.film()
            assert spp == spp0 == s.spp
            assert np.array_equal(sums[..., 3], sums0[..., 3]), "sample weights differ"
            err = _rel(sums[..., :3], sums0[..., :3])
            print(f"{s.name} {s.width}x{s.height}x{s.spp}: relMSE of the sums {err:.2e}")
            assert err < 1e-12
        # a second wavefront continues every scene's sample numbering
        photon_gpu.render_scenes_wavefront(rss, [2] * len(rss), max_bounces=10, estimator=est, seed=77)
        assert all(rs.film(with_sums=False)[2] == s.spp + 2 for s, rs in zip(sc, rss))
    finally:
        for rs in rss:
            rs.close()


@pytest.mark.gpu
def test_wavefront_rejects_filtered_films_and_duplicates(gpu_lib):
    import photon_gpu

    a = photon_gpu.RenderScene(scenes.cornell(32, 32, 4, 8))
    b = photon_gpu.RenderScene(scenes.cornell(32, 32, 4, 8))
    try:
        with pytest.raises(photon_gpu.PhotonGpuError):
            photon_gpu.render_scenes_wavefront([a, a], [4, 4], max_bounces=8)
        b.set_filter("bh")
        with pytest.raises(photon_gpu.PhotonGpuError):
            photon_gpu.render_scenes_wavefront([a, b], [4, 4], max_bounces=8)
        with pytest.raises(photon_gpu.PhotonGpuError):
            photon_gpu.render_scenes_wavefront([a], [0], max_bounces=8)
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_wavefront_autotune(gpu_lib):
    """The wavefront's launch shapes tuned on calibration wavefronts; the tuned batch still renders
    every scene's own paths."""
    import photon_gpu

    sc = _scenes()[:3]
    rss = [photon_gpu.RenderScene(s) for s in sc]
    try:
        t = photon_gpu.autotune_wavefront(rss, [s.spp for s in sc], max_bounces=10)
        print(f"wavefront autotune: {t}")
        assert t["trials"] > 0 and t["ms_tuned"] <= t["ms_default"]
        assert rss[0].launch()["capacity"] == t["capacity"]
        solo = []
        for s, rs in zip(sc, rss):
            rs.clear()
        photon_gpu.render_scenes_wavefront(rss, [s.spp for s in sc], max_bounces=10, seed=5)
        tuned = [rs.film()[1] for rs in rss]
        for s, rs in zip(sc, rss):
            rs.clear()
            rs.render(s.spp, max_bounces=10, seed=5)
            solo.append(rs.film()[1])
        for a, b in zip(tuned, solo):
            assert np.array_equal(a[..., 3], b[..., 3])
            assert _rel(a[..., :3], b[..., :3]) < 1e-12
    finally:
        for rs in rss:
            rs.close()
