"""Pins the oracle's CPU restatement (oracle/port/ph_port.cpp) to the reference.

The restatement is the checker the GPU path is compared with wherever the compiled reference is
not at hand (it is plain C++ and travels), so it must itself reproduce the reference's answers:

* closest hits and occlusion against the reference's TBinaryBvhIntersector answers (the same
  near-tie rule as the GPU traversal: a different primitive only where t agrees within 2 ulp);
* BSDF eval / pdf / sample against the reference's SurfaceOptics answers (bsdf_cases.npz);
* whole BNEEPT and BVPTDL images against the reference renders of images.npz, at fewer samples (4 x 4 block
  relMSE <= 1e-3 and per-channel means within 1 %, the bar of the GPU image tests);
* images through the reference's gaussian, Mitchell-Netravali and Blackman-Harris sample filters
  at full resolution (relMSE <= 1e-3; the same scene through the box filter is 3.5e-3 or more
  away from each of them, so the bar tells the filters apart).

CPU only; builds the library with ``make -f oracle/Makefile.port`` when it is missing.
"""

import dataclasses
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from test_trace_parity import ulp_diff

import scenes


@pytest.fixture(scope="module")
def port():
    from oracle.port import port as p

    if not os.path.exists(p.LIB):
        subprocess.run(["make", "-f", "oracle/Makefile.port"], cwd=ROOT, check=True,
                       stdout=subprocess.DEVNULL)
    p.load()
    return p


@pytest.mark.parametrize("name", ["hits_cornell.npz", "hits_sphere.npz"])
def test_port_hits_match_reference(port, name):
    d = dict(np.load(os.path.join(GOLDEN, name)))
    prim, t, bary, occ = port.trace(d["tris"], d["rays"])
    hit_ref = d["prim"] >= 0
    assert np.array_equal(prim >= 0, hit_ref)
    same = (prim == d["prim"]) & hit_ref
    near_tie = hit_ref & ~same & (ulp_diff(t, d["t"]) <= 2)
    assert np.all(same | near_tie | ~hit_ref)
    assert near_tie.sum() <= 0.06 * hit_ref.sum()
    assert np.array_equal(t[same].view(np.uint32), d["t"][same].view(np.uint32))
    assert np.array_equal(bary[same].view(np.uint32), d["bary"][same].view(np.uint32))
    assert np.array_equal(occ, d["occluded"])


def test_smoke_checker_on_port_hits(port):
    """smoke()'s closest-hit check accepts the port's answers on the Cornell fixture (including
    rays that start on a surface, hit at t = +0 where the reference reports -0), and rejects a
    wrong primitive, a hit turned into a miss and a t moved by 3 ulp."""
    import __graft_entry__ as entry

    d = dict(np.load(os.path.join(GOLDEN, "hits_cornell.npz")))
    prim, t, _, _ = port.trace(d["tris"], d["rays"])
    assert np.any((t == 0) & (d["t"] == 0) & np.signbit(d["t"]) & ~np.signbit(t))
    assert entry.hits_agree(prim, t, d["prim"], d["t"]).all()
    hit = np.flatnonzero((prim >= 0) & (prim == d["prim"]) & (t > 0))
    k = hit[0]
    bad = prim.copy()
    bad[k] = (prim[k] + 1) % d["tris"].shape[0]
    far = t.copy()
    far.view(np.int32)[k] += 3
    missed = prim.copy()
    missed[k] = -1
    assert not entry.hits_agree(missed, t, d["prim"], d["t"])[k]
    moved = entry.hits_agree(bad, far, d["prim"], d["t"])
    assert not moved[k] and moved.sum() == len(prim) - 1


def test_port_bsdf_matches_reference(port):
    d = np.load(os.path.join(GOLDEN, "bsdf_cases.npz"))
    cases, ref = d["cases"], d["out"]
    got = port.bsdf(cases, ref[:, 16:22])
    for k in (0, 4, 6):
        assert np.array_equal(got[:, k] > 0, ref[:, k] > 0), f"flag column {k} differs"
    ev, pd, sm = ref[:, 0] > 0, ref[:, 4] > 0, ref[:, 6] > 0
    assert np.allclose(got[ev, 1:4], ref[ev, 1:4], rtol=1e-5, atol=1e-7)
    assert np.allclose(got[pd, 5], ref[pd, 5], rtol=1e-5, atol=1e-7)
    assert np.allclose(got[sm, 7:10], ref[sm, 7:10], atol=2e-5)
    assert np.allclose(got[sm, 10:13], ref[sm, 10:13], rtol=1e-4, atol=1e-6)
    assert np.allclose(got[sm, 13], ref[sm, 13], rtol=1e-6)


# image name -> (scene factory, oracle spp)
IMAGES = {
    "cornell_bneept": (lambda spp: scenes.cornell(64, 64, spp, 8, "bneept"), 512),
    "cornell_bvptdl": (lambda spp: scenes.cornell(64, 64, spp, 8, "bvptdl"), 4096),
    "cornell_bneept_gaussian": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                                sample_filter="gaussian"), 1024),
    "cornell_bneept_mn": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                          sample_filter="mn"), 1024),
    "cornell_bneept_bh": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                          sample_filter="bh"), 1024),
    "cornell_glossy_bneept": (lambda spp: scenes.cornell_glossy(64, 64, spp, 8, "bneept"), 1024),
    "ggx_sphere_env_bneept": (lambda spp: scenes.ggx_sphere(level=3, width=64, height=64, spp=spp,
                                                            max_bounces=10), 512),
}


@pytest.mark.parametrize("name", list(IMAGES))
def test_port_image_matches_reference(port, name):
    import photon_gpu

    d = np.load(os.path.join(GOLDEN, "images.npz"))
    factory, spp = IMAGES[name]
    scene = factory(spp)
    estimator = {"bneept": 0, "bvpt": 1, "bvptdl": 2}[scene.estimator]
    filtered = scene.sample_filter != "box"
    img = port.render(photon_gpu.flatten_scene(scene), spp, scene.max_bounces, estimator, seed=3,
                      sample_filter=scene.sample_filter if filtered else None)
    ref = d[name]
    block = lambda a: a.reshape(16, 4, 16, 4, 3).mean(axis=(1, 3)).astype(np.float64)
    err = float(np.mean((block(img) - block(ref)) ** 2 / (block(ref) ** 2 + 1e-2)))
    means = img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1))
    assert err <= 1e-3, f"block relMSE {err:.3e}"
    assert np.all(np.abs(means - 1.0) < 0.01), means
    if filtered:
        full = float(np.mean((img.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + 1e-2)))
        assert full <= 1e-3, f"relMSE {full:.3e}"


def test_port_image_dome_matches_reference(port):
    """The lat-long sky-and-sun dome, rotated 60 degrees about +y: the restatement samples texels
    through the reference's 2D piecewise-constant distribution and uses its finite-dome densities."""
    import photon_gpu

    d = np.load(os.path.join(GOLDEN, "images.npz"))
    scene = scenes.ggx_sphere(level=3, width=64, height=64, spp=1024, max_bounces=10)   # constant dome in the flat arrays
    port.set_environment(scenes.sky_image(), ((0.0, 1.0, 0.0), 60.0))
    try:
        img = port.render(photon_gpu.flatten_scene(scene), 1024, 10, 0, seed=3)
    finally:
        port.set_environment()
    ref = d["ggx_sphere_envmap_bneept"]
    block = lambda a: a.reshape(16, 4, 16, 4, 3).mean(axis=(1, 3)).astype(np.float64)
    assert float(np.mean((block(img) - block(ref)) ** 2 / (block(ref) ** 2 + 1e-2))) <= 1e-3
    assert np.all(np.abs(img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1)) - 1.0) < 0.01)


def test_port_furnace_reference_and_exact_densities(port):
    """The grey furnace: with the reference's dome densities the restatement lands near the
    reference's biased render (0.512); with exact densities on the analytic 0.5."""
    import photon_gpu

    scene = scenes.furnace(512)
    ref = np.load(os.path.join(GOLDEN, "images.npz"))["furnace_bneept_ref"][12:20, 12:20].mean()
    try:
        port.set_environment(exact=False)
        biased = port.render(photon_gpu.flatten_scene(scene), 512, scene.max_bounces, 0, seed=3)[12:20, 12:20].mean()
        port.set_environment(exact=True)
        exact = port.render(photon_gpu.flatten_scene(scene), 512, scene.max_bounces, 0, seed=3)[12:20, 12:20].mean()
    finally:
        port.set_environment()
    assert abs(biased / ref - 1.0) < 1e-2, (biased, ref)
    assert abs(exact - 0.5) < 3e-3, exact
