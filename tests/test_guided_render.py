"""Learned path guiding inside the renderer.

* Unbiasedness: guiding changes the sampling density, never the expectation. A guided BNEEPT
  render (network trained online during the render) and a plain one of the same Cornell box agree
  in per-channel means within 1 % and in 4 x 4 block means within the bar of the image tests.
* Learning: over consecutive renders of the slit-light room the mean training loss (the weighted
  negative log-likelihood of the sampled directions, log 4 pi = 2.53 for a uniform density) falls
  well below its initial value.
"""

import numpy as np
import pytest

import scenes


def _rel_mse(x, ref, eps=1e-2):
    return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + eps)))


@pytest.mark.gpu
@pytest.mark.parametrize("depth", [1, 0])
def test_guided_render_is_unbiased(gpu_lib, depth):
    """depth 1 guides the surfaces the camera sees (the default), 0 every vertex."""
    import photon_gpu

    scene = scenes.cornell(32, 32, 1, 8)
    with photon_gpu.RenderScene(scene) as rs:
        rs.render(8192, max_bounces=8, seed=3)
        plain = rs.film()[0]
        rs.clear()
        rs.set_guiding(True, True, 0.5, 3e-3, 16384)
        rs.set_guiding_depth(depth)
        rs.render(8192, max_bounces=8, seed=5)
        guided = rs.film()[0]
        info = rs.guide_info()
    assert info["guided_vertices"] > 0
    means = guided.mean(axis=(0, 1)) / plain.mean(axis=(0, 1))
    block = lambda a: a.reshape(8, 4, 8, 4, 3).mean(axis=(1, 3))
    err = _rel_mse(block(guided), block(plain))
    print("guided/plain means", means, "block relMSE", err, "loss", info["loss"])
    assert np.all(np.abs(means - 1.0) < 0.01), means
    assert err < 2e-3, err


@pytest.mark.gpu
def test_guiding_network_learns_the_slit_room(gpu_lib):
    import photon_gpu

    scene = scenes.slit_room(64, 64, 1, 10, num_boxes=2000)
    losses = []
    with photon_gpu.RenderScene(scene) as rs:
        rs.set_guiding(True, True, 0.5, 3e-3, 16384)
        for k in range(8):
            rs.clear()
            rs.render(64, max_bounces=10, seed=100 + k)
            losses.append(rs.guide_info()["loss"])
    print("mean training loss per render", np.round(losses, 3))
    assert np.all(np.isfinite(losses))
    assert losses[0] > 2.0
    assert np.mean(losses[-4:]) < losses[0] - 0.25, losses
