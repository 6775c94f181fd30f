"""The benchmarked workloads are the configurations they stand for.

bench.py renders five workloads built by photon-v2_b200/scenes.py; their throughput and error
numbers mean something only if the builders produce the configured scenes. Each test checks one
builder against its configuration: triangle counts, materials and their parameter ranges, lights,
resolution, samples per pixel and bounce cap.

* C1 Cornell box: 5 wall quads, 2 rotated boxes, 1 ceiling quad light of radiance (17, 12, 4) in
  a 555-unit box (36 triangles), albedos 0.73 / (0.65, 0.05, 0.05) / (0.12, 0.45, 0.15), 40 degree
  field of view, 256 x 256, 64 spp, depth 8.
* C2: icosphere subdivided to 20 * 4^8 = 1,310,720 triangles, radially displaced by at most 5 % of
  the radius, on a 2-triangle ground; GGX conductors with roughness in [0.05, 0.5] and F0 in
  [0.5, 1]; 2 quad lights and a constant environment of 0.1; 1024 x 1024, 256 spp, depth 10.
* C3: 64 scenes of 1k-500k triangles, resolutions 128-1024 squared, 16-256 spp, 1-4 quad lights,
  Lambertian and GGX material groups about half and half.
* C4 slit room: 10 x 10 x 4 room, 2M triangles of boxes, one 1 x 1 light behind a wall with a
  0.05-wide slit, 70 % Lambertian and 30 % GGX dielectric (IOR 1.5, roughness 0.1), 1024 x 1024.
* C5 city: 447^2 buildings with lognormal(2, 0.6) heights, each 108 triangles (21.6M with the
  ground and lights), 10,000 emissive quads of lognormal(sigma 1) power, GGX roughness in
  [0.02, 0.8], 1920 x 1080, 1024 spp, depth 12. The full city is counted by its formula and
  its statistics are checked on a 100 x 100 grid from the same generator.
"""

import numpy as np
import pytest

import scenes


def _tri_count(sc):
    return sum(g.tris.shape[0] for g in sc.groups)


def _emitters(sc):
    return [g for g in sc.groups if g.radiance is not None]


def test_c1_cornell():
    sc = scenes.cornell()
    assert (sc.width, sc.height, sc.spp, sc.max_bounces, sc.fov_deg) == (256, 256, 64, 8, 40.0)
    assert _tri_count(sc) == 36
    lights = _emitters(sc)
    assert len(lights) == 1 and lights[0].tris.shape[0] == 2 and lights[0].radiance == (17.0, 12.0, 4.0)
    albedos = {g.material.albedo for g in sc.groups if g.radiance is None}
    assert albedos == {(0.73, 0.73, 0.73), (0.65, 0.05, 0.05), (0.12, 0.45, 0.15)}
    v = np.concatenate([g.tris.reshape(-1, 3) for g in sc.groups])
    assert v.min() >= 0.0 and v.max() <= 555.0


def test_c2_displaced_ggx_sphere():
    sc = scenes.ggx_sphere(level=8)
    assert (sc.width, sc.height, sc.spp, sc.max_bounces) == (1024, 1024, 256, 10)
    assert sc.env_radiance == (0.1, 0.1, 0.1)
    conductors = [g for g in sc.groups if g.material.kind == "conductor"]
    sphere = np.concatenate([g.tris for g in conductors])
    assert sphere.shape[0] == 20 * 4 ** 8 == 1_310_720
    assert _tri_count(sc) == 1_310_726   # + ground (2) + two quad lights (4)
    assert len(conductors) == 64
    assert all(0.05 <= g.material.roughness <= 0.5 for g in conductors)
    assert all(0.5 <= c <= 1.0 for g in conductors for c in g.material.f0)
    # vertices on the sphere of radius 1 centred 1.05 above the ground, displaced by at most 5 %
    p = sphere.reshape(-1, 3).astype(np.float64) - np.array([0.0, 1.05, 0.0])
    r = np.linalg.norm(p, axis=1)
    assert r.min() >= 0.95 - 1e-5 and r.max() <= 1.05 + 1e-5
    assert r.std() > 0.005   # actually displaced
    assert len(_emitters(sc)) == 2


@pytest.mark.parametrize("index", [0, 1, 2, 3, 30, 31, 62, 63])
def test_c3_batched_scene(index):
    sc = scenes.batch_scene(index)
    assert 128 <= sc.width == sc.height <= 1024
    assert 16 <= sc.spp <= 256
    assert 1 <= len(_emitters(sc)) <= 4
    n = _tri_count(sc) - 2 - 2 * len(_emitters(sc))   # without the ground and the lights
    assert 1_000 * 0.98 <= n <= 500_000 if index % 2 == 0 else 1_280 <= n <= 327_680
    kinds = {g.material.kind for g in sc.groups if g.radiance is None}
    assert kinds <= {"matte", "conductor"}


def test_c3_material_mix_is_half_and_half():
    """Over the 64 scenes the non-ground material groups are Lambertian or GGX with probability 1/2."""
    kinds = []
    for index in range(0, 64, 4):
        sc = scenes.batch_scene(index)
        kinds += [g.material.kind for g in sc.groups[:-1 - len(_emitters(sc))] if g.radiance is None]
    frac = np.mean([k == "matte" for k in kinds])
    assert 0.3 <= frac <= 0.7, frac


def test_c4_slit_room():
    sc = scenes.slit_room()
    assert (sc.width, sc.height) == (1024, 1024)
    assert _tri_count(sc) == 2_000_042   # 166,667 boxes + room shell, dividing wall and light
    lights = _emitters(sc)
    assert len(lights) == 1
    lv = lights[0].tris.reshape(-1, 3)
    assert np.allclose(lv.max(0) - lv.min(0), [0.0, 1.0, 1.0])   # a 1 x 1 quad
    v = np.concatenate([g.tris.reshape(-1, 3) for g in sc.groups])
    assert np.allclose(v.min(0), [0.0, 0.0, 0.0]) and np.allclose(v.max(0), [10.0, 4.0, 10.0])
    glass = [g for g in sc.groups if g.material.kind == "dielectric"]
    matte_boxes = sc.groups[1]
    assert len(glass) == 1
    g = glass[0].material
    assert (g.roughness, g.ior_outer, g.ior_inner) == (0.1, 1.0, 1.5)
    frac = glass[0].tris.shape[0] / (glass[0].tris.shape[0] + matte_boxes.tris.shape[0])
    assert 0.29 <= frac <= 0.31, frac
    # the slit: the dividing wall at x = 8 leaves z in (4.975, 5.025) open over the full height
    wall = sc.groups[0].tris.reshape(-1, 3)
    at_wall = wall[np.abs(wall[:, 0] - 8.0) < 0.06]
    gap = np.sort(np.unique(np.round(at_wall[:, 2], 4)))
    assert 4.975 in gap and 5.025 in gap
    assert not np.any((at_wall[:, 2] > 4.975 + 1e-4) & (at_wall[:, 2] < 5.025 - 1e-4))


def test_c5_city_counts_and_statistics():
    blocks, lights = 447, 10_000
    assert blocks ** 2 * 108 + 2 + 2 * lights == 21_599_374   # the full city (bench: 21,599,374)
    sc = scenes.city(blocks=100, num_lights=lights)
    assert (sc.width, sc.height, sc.spp, sc.max_bounces) == (1920, 1080, 1024, 12)
    assert _tri_count(sc) == 100 ** 2 * 108 + 2 + 2 * lights
    conductors = [g for g in sc.groups if g.material.kind == "conductor"]
    assert all(0.02 <= g.material.roughness <= 0.8 for g in conductors)
    # building heights: the top of every tessellated box, lognormal(mu 2, sigma 0.6)
    boxes = np.concatenate([g.tris for g in conductors]).reshape(-1, 108, 3, 3)
    h = np.log(boxes[:, :, :, 1].max(axis=(1, 2)).astype(np.float64))
    assert abs(h.mean() - 2.0) < 0.03 and abs(h.std() - 0.6) < 0.03
    em = _emitters(sc)
    assert len(em) == lights
    power = np.log(np.array([np.mean(g.radiance) for g in em]))
    assert abs(power.std() - 1.0) < 0.05
