"""Light selection and NEE densities against the reference's power-favouring emitter sampler.

Fixtures (tests/golden/make_golden.py, `lights` part) hold, for 3, 100 and 10,000 area emitters of
lognormal power (quads, single triangles and 2 x 2-tessellated quads), what the reference's own
classes answer:

* `flux`: Emitter::calcRadiantFluxApprox of each emitter, the weight ESPowerFavoring::update gives
  it (Engine/Source/Core/Emitter/Sampler/ESPowerFavoring.cpp:41-49; colour energy x area x pi,
  DiffuseSurfaceEmitter.cpp:55-86, summed over a group, GroupedDiffuseSurfaceEmitter.cpp:110-120);
* `pmf`: the sampler's pick probability, TPwcDistribution1D::pdfDiscrete -- the difference of two
  entries of a float32 CDF, so it carries that CDF's rounding: up to about one float32 ulp of 1
  (1.2e-7) absolute, which for the smallest of 10,000 emitters is most of its value (one of them
  rounds to 0 there);
* `pdf_w`: ESPowerFavoring::calcDirectPdf for (receiving point, point on a light triangle) pairs,
  and `emitter_pdf_w` the emitter's own density without the pick (SurfaceEmitter.cpp:37-61).

Bars: the GPU pick probability equals flux / sum(flux) within 1e-6 relative and the reference's
realised pmf within 2e-7 absolute; the device alias table realises the GPU pmf within 1e-6
relative; the NEE density equals the reference emitter density x flux / sum(flux) within
1e-5 + 3e-7 / cos relative (cos: the cosine at the light point, whose float32 error of a few ulps
of 1 both sides share, so grazing light points carry it amplified), the reference's own pdf within
the same bar wherever its pmf is not rounded (relative CDF error below 1e-6), and is exactly 0
wherever the reference's is (back-facing light points).
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN

import scenes

COUNTS = (3, 100, 10_000)


def _load(count):
    return dict(np.load(os.path.join(GOLDEN, f"lights_{count}.npz")))


def _scene(d):
    """A flat scene of exactly the fixture's emitters, in order (emitter k = group k)."""
    first = d["group_first"]
    groups = [scenes.MeshGroup(d["tris"][first[k]:first[k + 1]], scenes.BLACK,
                               radiance=tuple(float(x) for x in d["radiance"][k]))
              for k in range(len(first) - 1)]
    return scenes.Scene("lights", 8, 8, 1, 2, cam_pos=(0.0, 0.0, -200.0), cam_dir=(0.0, 0.0, 1.0),
                        cam_up=(0.0, 1.0, 0.0), fov_deg=40.0, groups=groups)


@pytest.mark.parametrize("count", COUNTS)
def test_reference_pmf_is_its_flux_share(count):
    """The reference's realised pmf is flux / sum(flux) up to its float32 CDF's rounding."""
    d = _load(count)
    flux = d["flux"].astype(np.float64)
    assert flux.shape == (count,) and np.all(flux > 0)
    ideal = flux / flux.sum()
    assert np.max(np.abs(d["pmf"] - ideal)) <= 2e-7
    assert d["hit"].all()
    # the sampler's density is the emitter's density times the realised pmf
    owner = np.searchsorted(d["group_first"], d["prim"], side="right") - 1
    has = d["pdf_w"] > 0
    np.testing.assert_allclose(d["pdf_w"][has], d["emitter_pdf_w"][has] * d["pmf"][owner[has]], rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("count", COUNTS)
def test_gpu_pick_probabilities_match_reference(gpu_lib, count):
    import photon_gpu

    d = _load(count)
    flux = d["flux"].astype(np.float64)
    ideal = flux / flux.sum()
    with photon_gpu.RenderScene(_scene(d)) as rs:
        pmf, alias_pmf = rs.light_pmf()
    assert pmf.shape == (count,)
    rel = np.abs(pmf.astype(np.float64) - ideal) / ideal
    print(f"{count} emitters: max rel |pmf - flux share| {rel.max():.2e}, "
          f"max |pmf - reference pmf| {np.abs(pmf - d['pmf']).max():.2e}, "
          f"max rel |alias - pmf| {np.max(np.abs(alias_pmf - pmf) / pmf):.2e}")
    assert rel.max() <= 1e-6
    assert np.abs(pmf.astype(np.float64) - d["pmf"]).max() <= 2e-7
    np.testing.assert_allclose(alias_pmf, pmf.astype(np.float64), rtol=1e-6)
    assert abs(alias_pmf.sum() - 1.0) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("count", COUNTS)
def test_gpu_nee_densities_match_reference(gpu_lib, count):
    import photon_gpu

    d = _load(count)
    flux = d["flux"].astype(np.float64)
    ideal = flux / flux.sum()
    owner = np.searchsorted(d["group_first"], d["prim"], side="right") - 1
    with photon_gpu.RenderScene(_scene(d)) as rs:
        pdf = rs.light_pdf(d["targets"], d["point"], d["prim"]).astype(np.float64)
    ref_zero = d["emitter_pdf_w"] == 0
    assert np.all(pdf[ref_zero] == 0.0), "density where the reference's light point does not face the target"
    has = ~ref_zero
    # The density divides by the cosine at the light point; both sides compute that cosine in
    # float32 to a few ulps of 1, so at grazing light points its relative error grows as 1 / cos.
    tri = d["tris"][d["prim"]].astype(np.float64)
    nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    to_target = d["targets"].astype(np.float64) - d["point"]
    cos = np.abs((nrm * to_target).sum(1)) / np.linalg.norm(to_target, axis=1)
    tol = 1e-5 + 3e-7 / np.maximum(cos, 1e-12)
    want = d["emitter_pdf_w"][has] * ideal[owner[has]]
    rel = np.abs(pdf[has] - want) / want
    print(f"{count} emitters: {has.sum()} densities, max rel error {rel.max():.2e}, "
          f"max error / bar {np.max(rel / tol[has]):.2f}, smallest cosine {cos[has].min():.1e}")
    assert np.all(rel <= tol[has])
    # against the reference's own density where its pmf is not visibly rounded
    exact = has & (np.abs(d["pmf"][owner] - ideal[owner]) <= 1e-6 * ideal[owner])
    rel_ref = np.abs(pdf[exact] - d["pdf_w"][exact]) / d["pdf_w"][exact]
    assert np.all(rel_ref <= tol[exact])


def _quad_lights(radiances):
    """Equal unit quads in a row, each its own area emitter of grey radiance r (so that their
    fluxes stand in the ratio of the radiances)."""
    groups = []
    for k, r in enumerate(radiances):
        x = 3.0 * k
        quad = np.array([[[x, 0, 0], [x + 1, 0, 0], [x + 1, 1, 0]],
                         [[x, 0, 0], [x + 1, 1, 0], [x, 1, 0]]], np.float32)
        groups.append(scenes.MeshGroup(quad, scenes.BLACK, radiance=(float(r), float(r), float(r))))
    return scenes.Scene("quad lights", 8, 8, 1, 2, cam_pos=(0.0, 0.0, -20.0), cam_dir=(0.0, 0.0, 1.0),
                        cam_up=(0.0, 1.0, 0.0), fov_deg=40.0, groups=groups)


@pytest.mark.gpu
def test_gpu_pick_never_takes_zero_power_emitters(gpu_lib):
    """The reference's PiecewiseConstantDistribution1DTest.ContinuousSampleInRange
    (Engine/EngineTest/Source/Math/Random/distribution_test.cpp:21-44): of the weights
    {0, 0, 1, 0, 2, 3, 0}, entries 0, 1, 3 and 6 are never sampled. As light selection: their pick
    probability and the probability the device alias table realises for them are exactly 0, and
    the others take 1/6, 2/6 and 3/6 (1e-6 relative)."""
    import photon_gpu

    weights = np.array([0, 0, 1, 0, 2, 3, 0], np.float64)
    with photon_gpu.RenderScene(_quad_lights(weights)) as rs:
        pmf, alias_pmf = rs.light_pmf()
    zero = weights == 0
    assert np.all(pmf[zero] == 0.0) and np.all(alias_pmf[zero] == 0.0)
    np.testing.assert_allclose(pmf[~zero], weights[~zero] / 6.0, rtol=1e-6)
    np.testing.assert_allclose(alias_pmf[~zero], weights[~zero] / 6.0, rtol=1e-6)


@pytest.mark.gpu
def test_gpu_pick_of_all_zero_powers_is_uniform(gpu_lib):
    """The reference's PiecewiseConstantDistribution1DTest.CornerCases (distribution_test.cpp:
    80-92): weights that are all zero give the uniform distribution, 1/3 each for three; the same
    for three emitters of zero radiance (the device table realises it exactly)."""
    import photon_gpu

    with photon_gpu.RenderScene(_quad_lights([0.0, 0.0, 0.0])) as rs:
        pmf, alias_pmf = rs.light_pmf()
    np.testing.assert_allclose(pmf, 1.0 / 3.0, rtol=1e-7)
    assert np.all(alias_pmf == 1.0 / 3.0)
