"""Image parity of the GPU estimators with the reference CPU renderer, plus analytic checks.

Renders go through the Photon C API of this library (SDL text -> phLoadCommands -> phUpdate ->
phRender -> phAquireFrameRaw), exactly as a reference user would drive it. References:

* images.npz -- renders of the same SDL by the reference's own EqualSamplingRenderer +
  BNEEPTEstimator / BVPTEstimator / BVPTDLEstimator (tests/golden/make_golden_images.py, 64 x 64,
  4096-8192 spp),
  in the reference's default iterative surface refinement and, for two scenes, in its empirical
  and manual modes (the reference's EngineConfig.ini on its side, phGpuSetSurfaceRefine on ours).
  The bar is an image tolerance of relMSE <= 1e-3, relMSE being the mean over pixels
  and channels of (x - ref)^2 / (ref^2 + 1e-2). Both images carry Monte Carlo noise, which the
  bound includes. BNEEPT images meet it at full resolution; BVPT and BVPTDL (no light sampling, a
  small light) are noise-dominated at these sample counts, so it is held to the bar on 4 x 4 block means
  (16 x fewer noise, same expectation) and to a looser full-resolution bound. The glossy scene's
  caustics through the glass box are noisy at any spp, so its GPU side renders 16384 spp: the
  relMSE of two independent renders is the sum of their variances, and this keeps the GPU's
  share below the reference image's own. Per-channel image means must agree within 1 %
  everywhere.
* the furnace known answer (the reference's Main/RenderTest/tests/test_gray_furnace_box.py:
  |mean - 0.5| < 1e-3): a convex Lambertian object of albedo 0.5 under a uniform environment of
  radiance 1 reflects exactly 0.5;
* unit radiance (Main/RenderTest/tests/test_fullscreen_unit_radiance.py): a camera enclosed by
  emitters of radiance 1 sees exactly 1 in every pixel.
"""

import dataclasses
import os

import numpy as np
import pytest

from conftest import GOLDEN

import scenes

IMAGES = os.path.join(GOLDEN, "images.npz")

# workload name -> (scene factory, GPU spp)
WORKLOADS = {
    "cornell_bneept": (lambda spp: scenes.cornell(64, 64, spp, 8, "bneept"), 4096),
    "cornell_bvpt": (lambda spp: scenes.cornell(64, 64, spp, 8, "bvpt"), 4096),
    "cornell_bvptdl": (lambda spp: scenes.cornell(64, 64, spp, 8, "bvptdl"), 4096),
    # lat-long image dome, importance-sampled by its luminance x sin(theta), rotated dome
    "ggx_sphere_envmap_bneept": (lambda spp: dataclasses.replace(
        scenes.ggx_sphere(level=3, width=64, height=64, spp=spp, max_bounces=10),
        env_radiance=None, env_image=scenes.sky_image(), env_rotation=((0.0, 1.0, 0.0), 60.0)), 8192),
    "cornell_glossy_bneept": (lambda spp: scenes.cornell_glossy(64, 64, spp, 8, "bneept"), 16384),
    "ggx_sphere_env_bneept": (lambda spp: scenes.ggx_sphere(level=3, width=64, height=64, spp=spp,
                                                            max_bounces=10), 4096),
    # the reference's other surface-refine modes (RefineMode in its EngineConfig.ini)
    "cornell_glossy_bneept_empirical": (lambda spp: scenes.cornell_glossy(64, 64, spp, 8, "bneept"), 16384,
                                        "empirical"),
    "ggx_sphere_bneept_manual": (lambda spp: scenes.ggx_sphere(level=3, width=64, height=64, spp=spp,
                                                               max_bounces=10), 4096, "manual"),
    # the reference's other sample filters (HdrRgbFilm::addRgbSample through SampleFilter)
    "cornell_bneept_gaussian": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                                sample_filter="gaussian"), 4096),
    "cornell_bneept_mn": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                          sample_filter="mn"), 4096),
    "cornell_bneept_bh": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                          sample_filter="bh"), 4096),
}


def rel_mse(x, ref, eps=1e-2):
    return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + eps)))


def render_via_c_api(scene, tmp_path, seed=1, refine_mode="iterative", dome_pdf="reference", mesh_format="text"):
    import photon_gpu

    p2 = tmp_path / "scene.p2"
    p2.write_text(scenes.to_sdl(scene, mesh_format=mesh_format))
    if mesh_format == "ply":
        scenes.write_meshes(scene, str(tmp_path))
    scenes.write_env(scene, str(tmp_path))
    with photon_gpu.PhotonEngine() as eng:
        eng.set_working_directory(str(tmp_path))
        assert eng.load_file(str(p2)), eng.errors()
        eng.set_max_bounces(scene.max_bounces)
        eng.set_seed(seed)
        eng.set_surface_refine(refine_mode)
        eng.set_dome_pdf(dome_pdf)
        eng.update()
        eng.render()
        img = eng.frame()
        info = eng.info()
    assert info["paths"] == scene.width * scene.height * scene.spp
    return img, info


# The benchmarked configurations' geometry at reduced resolution (tests/golden/make_golden_images.py):
# name -> (scene factory, reference spp, full-resolution relMSE bar or None). The meshes reach the
# GPU as binary PLY files through geometry(ply) (the reference parsed the same triangles as SDL text).
LARGE_WORKLOADS = {
    # 1,310,726 triangles, 2 quad lights + environment, GGX in 64 groups, depth 10, 64 x 64
    "c2_ggx1m_bneept": (lambda spp: scenes.ggx_sphere(level=8, width=64, height=64, spp=spp, max_bounces=10),
                        65536, 1e-3),
    # 2,000,042 triangles, light through a 0.05-wide slit, 30 % rough glass boxes, depth 10, 32 x 32
    "slit_room_bneept": (lambda spp: scenes.slit_room(32, 32, spp, 10), 262144, None),
    # the same room with every box Lambertian (no caustics), and with its glass at depth 2
    "slit_room_matte_bneept": (lambda spp: scenes.slit_room(32, 32, spp, 10, glass_fraction=0.0), 16384, None),
    "slit_room_depth2_bneept": (lambda spp: scenes.slit_room(32, 32, spp, 2), 262144, None),
    # 174,802 triangles, 1,000 lights of lognormal radiance, GGX roughness 0.02-0.8, depth 12, 64 x 64
    "city_tile_bneept": (lambda spp: scenes.city(64, 64, spp, 12, blocks=40, num_lights=1000), 16384, None),
}


def test_golden_images_present():
    d = np.load(IMAGES)
    for name in WORKLOADS:
        assert d[name].shape == (64, 64, 3)
        assert np.all(np.isfinite(d[name])) and d[name].mean() > 0
    for name, (factory, _, _) in LARGE_WORKLOADS.items():
        sc = factory(1)
        assert d[name].shape == (sc.height, sc.width, 3)
        assert np.all(np.isfinite(d[name])) and d[name].mean() > 0


def _block(a, k):
    h, w, c = a.shape
    return a.reshape(h // k, k, w // k, k, c).mean(axis=(1, 3))


def _mean_spread(scene, spp, seeds=8):
    """Relative standard deviation, per channel, of the image mean of spp-sample renders over
    seeds: the noise of a reference render's mean, measured on the GPU."""
    import photon_gpu

    with photon_gpu.RenderScene(scene) as rs:
        means = []
        for k in range(seeds):
            rs.clear()
            rs.render(spp, max_bounces=scene.max_bounces, seed=500 + k)
            means.append(rs.film(with_sums=False)[0].mean(axis=(0, 1)))
    m = np.asarray(means, np.float64)
    return m.std(axis=0, ddof=1) / m.mean(axis=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(LARGE_WORKLOADS))
def test_benchmarked_geometry_matches_reference(gpu_lib, tmp_path, name):
    """Image parity on the geometry of the benchmarked configurations: the 1M-triangle GGX scene,
    the 2M-triangle slit room with its glass, and a 1,000-light city tile, against reference
    renders of 16,384-65,536 spp. The GPU side renders 4 x the reference's samples, so the
    difference is mostly the reference's own noise. A systematic difference (bias) survives
    averaging, noise does not: relMSE of 8 x 8-block means <= 1e-3 (64 x less noise) and
    per-channel means within 1 %, or within 4 standard deviations of the difference where the
    image mean itself is that noisy: the spread of the mean over 8 GPU renders at the reference's
    spp gives the reference's (sigma) and the GPU image's (sigma / 2). That is the case in the slit
    room with its glass, where rare paths through glass boxes lit through the slit carry most of
    the error (sigma ~2 % at 65,536 spp); its glass-free and depth-2 variants hold the 1 % bar.
    Where the reference render is converged enough (the 1M-triangle scene) relMSE <= 1e-3 holds
    at full resolution too; in the slit room and the city, light found through a 5 cm slit or
    from 1,000 small lights on near-mirror GGX leaves a 16K-65K-spp reference with per-pixel
    noise above that (its full-resolution relMSE is printed)."""
    d = np.load(IMAGES)
    ref = d[name]
    factory, spp, full_bar = LARGE_WORKLOADS[name]
    assert spp == int(d[name + "__spp"])
    scene = factory(4 * spp)
    assert scene.max_bounces == int(d[name + "__bounces"])
    img, _ = render_via_c_api(scene, tmp_path, mesh_format="ply")
    err = rel_mse(img, ref)
    err_blocks = rel_mse(_block(img, 8), _block(ref, 8))
    means = img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1))
    sigma = _mean_spread(factory(1), spp)
    bar = np.maximum(0.01, 4.0 * sigma * np.sqrt(1.0 + 1.0 / 4.0))
    print(f"{name}: relMSE {err:.2e}, 8x8-block relMSE {err_blocks:.2e}, mean ratio {means}, "
          f"relative sigma of a {spp}-spp mean {sigma}, bar {bar}")
    assert err_blocks <= 1e-3, f"block relMSE {err_blocks:.3e}"
    assert np.all(np.abs(means - 1.0) < bar), f"channel means differ: {means} (bar {bar})"
    if full_bar is not None:
        assert err <= full_bar, f"relMSE {err:.3e}"


@pytest.mark.gpu
def test_c2_error_at_bench_spp(gpu_lib, tmp_path):
    """The error the benchmarked render carries: the 1M-triangle GGX scene at the bench's 256 spp
    against the 65,536-spp reference render (at 64 x 64), relMSE as the bench line states it.
    The error of an n-spp render falls as 1/n, which gives the spp that reaches relMSE 1e-3."""
    ref = np.load(IMAGES)["c2_ggx1m_bneept"]
    img, _ = render_via_c_api(scenes.ggx_sphere(level=8, width=64, height=64, spp=256, max_bounces=10), tmp_path,
                              mesh_format="ply")
    err = rel_mse(img, ref)
    print(f"c2 at 256 spp: relMSE {err:.3e} against the 65,536-spp reference; 1e-3 at ~{256 * err / 1e-3:.0f} spp")
    # Monte Carlo error at 256 spp on this scene: well under 1e-2, and the means agree within 1 %
    assert err < 1e-2
    assert np.all(np.abs(img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1)) - 1.0) < 0.01)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(WORKLOADS))
def test_image_matches_reference(gpu_lib, tmp_path, name):
    d = np.load(IMAGES)
    ref = d[name]
    factory, spp, *mode = WORKLOADS[name]
    scene = factory(spp)
    assert scene.max_bounces == int(d[name + "__bounces"])
    img, _ = render_via_c_api(scene, tmp_path, refine_mode=mode[0] if mode else "iterative")
    err = rel_mse(img, ref)
    block = lambda a: a.reshape(16, 4, 16, 4, 3).mean(axis=(1, 3))
    err_blocks = rel_mse(block(img), block(ref))
    means = img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1))
    print(f"{name}: relMSE {err:.2e}, 4x4-block relMSE {err_blocks:.2e}, mean ratio {means}")
    assert err_blocks <= 1e-3, f"block relMSE {err_blocks:.3e}"
    assert err <= (1e-3 if scene.estimator == "bneept" else 2e-2), f"relMSE {err:.3e}"
    assert np.all(np.abs(means - 1.0) < 0.01), f"channel means differ: {means}"


@pytest.mark.gpu
def test_ply_meshes_match_reference(gpu_lib, tmp_path):
    """The Cornell box with every mesh loaded from binary PLY files (geometry(ply)) renders the
    reference's Cornell image (the reference loads the same files: GPlyPolygonMesh)."""
    ref = np.load(IMAGES)["cornell_bneept"]
    img, _ = render_via_c_api(scenes.cornell(64, 64, 4096, 8, "bneept"), tmp_path, mesh_format="ply")
    assert rel_mse(img, ref) <= 1e-3
    assert np.all(np.abs(img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1)) - 1.0) < 0.01)


@pytest.mark.gpu
@pytest.mark.parametrize("estimator,sample_filter", [("bneept", "box"), ("bvpt", "box"), ("bneept", "gaussian"),
                                                     ("bneept", "mn"), ("bneept", "bh")])
def test_furnace(gpu_lib, tmp_path, estimator, sample_filter):
    # exact dome densities: the analytic answer. With a filter, light found by NEE at a path's last
    # vertex reaches the film from the traversal kernel, the rest from the shading kernel: both
    # must weight it like the sample's W.
    img, _ = render_via_c_api(scenes.furnace(1024, estimator, sample_filter), tmp_path, dome_pdf="exact")
    # the central pixels see only the sphere; the corners see only the environment
    centre = img[12:20, 12:20]
    assert abs(centre.mean() - 0.5) < 1e-3, centre.mean()
    assert np.allclose(img[0, 0], 1.0) and np.allclose(img[-1, -1], 1.0)


@pytest.mark.gpu
def test_furnace_with_the_reference_dome_densities(gpu_lib, tmp_path):
    """The reference's own densities on its finite dome sphere overestimate the furnace (its render
    gives 0.512, not 0.5, at the sphere's centre pixels); by default the GPU renderer computes
    them the same way and must land near the reference's render, not near 0.5. This dome is only
    1.75 x the sphere's radius, the most the densities deviate; the GPU render comes out 0.45 %
    above the reference's (0.514), against 2.4 % for the exact densities, so the bar is 1 %."""
    ref = np.load(IMAGES)["furnace_bneept_ref"][12:20, 12:20].mean()
    assert ref > 0.505
    img, _ = render_via_c_api(scenes.furnace(4096), tmp_path)
    centre = img[12:20, 12:20].mean()
    assert abs(centre / ref - 1.0) < 1e-2, (centre, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("sample_filter", ["box", "gaussian", "mn", "bh"])
def test_unit_radiance(gpu_lib, tmp_path, sample_filter):
    walls = scenes.boxes_axis_aligned(np.array([[-10.0, -10.0, -10.0]]), np.array([[10.0, 10.0, 10.0]]))
    walls = walls[:, [0, 2, 1]]   # flip winding so the faces (and their emission) point inwards
    groups = [scenes.MeshGroup(walls, scenes.Material("matte", albedo=(0.0, 0.0, 0.0)), radiance=(1.0, 1.0, 1.0))]
    scene = scenes.Scene("unit", 16, 16, 16, 10000, cam_pos=(0.0, 0.0, 0.0), cam_dir=(0.0, 0.0, 1.0),
                         cam_up=(0.0, 1.0, 0.0), fov_deg=60.0, groups=groups, sample_filter=sample_filter)
    img, _ = render_via_c_api(scene, tmp_path)
    assert np.allclose(img, 1.0, atol=1e-6), (img.min(), img.max())


@pytest.mark.gpu
@pytest.mark.parametrize("sample_filter", ["box", "bh"])
def test_developed_frame_is_sums_over_weight(gpu_lib, sample_filter):
    """The GPU develop equals RGB / W of the FP64 sums, rounded once to FP32, bit for bit; the box
    filter's W is the sample count."""
    import photon_gpu

    scene = scenes.cornell(32, 24, 8, 8, "bneept")
    with photon_gpu.RenderScene(scene) as rs:
        rs.set_filter(sample_filter)
        rs.render(8, max_bounces=8, seed=5)
        rs.render(3, max_bounces=8, seed=5, first_sample=8)
        rgb, sums, spp = rs.film()
    assert spp == 11 and rgb.shape == (24, 32, 3) and sums.shape == (24, 32, 4)
    w = sums[..., 3:4]
    assert np.all(w > 0)
    if sample_filter == "box":
        assert np.all(w == 11.0)
    want = (sums[..., :3] * (1.0 / w)).astype(np.float32)
    assert np.array_equal(rgb.view(np.uint32), want.view(np.uint32))
