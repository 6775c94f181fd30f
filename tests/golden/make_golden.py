"""Generates the golden fixtures of the parity tests by running the reference's own code.

Run in the build container, where the reference sources exist and the oracle has been built
(``make -f oracle/Makefile.ref REF=<reference sources> -j8``):

    python tests/golden/make_golden.py

It writes, next to this script:
  hits_cornell.npz, hits_sphere.npz   rays + closest-hit primitive/t/barycentrics + occlusion,
                                      computed by the reference's TBinaryBvhIntersector over
                                      PTriangles (oracle/_ref/ph_ref_golden hits)
  bsdf_cases.npz                      BSDF eval/pdf/sample answers of LambertianReflector,
                                      OpaqueMicrofacet and TranslucentMicrofacet
                                      (oracle/_ref/ph_ref_golden bsdf)
  c2_hits.npz                         closest hits / occlusion of ~32K rays on the benchmarked
                                      1.31M-triangle scene (inputs regenerated by the test)
  lights_3/100/10000.npz              ESPowerFavoring pick probabilities and NEE densities over
                                      3, 100 and 10,000 area emitters of lognormal power
                                      (oracle/_ref/ph_ref_golden lights)
All inputs are seeded, so re-running reproduces the files bit for bit.
"""

from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "photon-v2_b200"))

import scenes  # noqa: E402

GOLDEN_TOOL = os.path.join(ROOT, "oracle", "_ref", "ph_ref_golden")


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def camera_rays(scene: scenes.Scene, nx: int, ny: int, rng) -> np.ndarray:
    """Pinhole rays of the scene's camera through jittered raster positions (forward direction)."""
    pos = np.array(scene.cam_pos, np.float64)
    fwd = _unit(np.array(scene.cam_dir, np.float64))
    up = np.array(scene.cam_up, np.float64)
    z = -fwd
    x = _unit(np.cross(up, z))
    y = np.cross(z, x)
    aspect = scene.width / scene.height
    half_w = np.tan(np.radians(scene.fov_deg) * 0.5)
    half_h = half_w / aspect
    gx, gy = np.meshgrid((np.arange(nx) + rng.random(nx)) / nx, (np.arange(ny) + rng.random(ny)) / ny)
    sx = (2 * gx.ravel() - 1) * half_w
    sy = (2 * gy.ravel() - 1) * half_h
    d = _unit(sx[:, None] * x + sy[:, None] * y - z)
    o = np.broadcast_to(pos, d.shape)
    return make_rays(o, d, 0.0, np.finfo(np.float32).max)


def make_rays(o, d, tmin, tmax) -> np.ndarray:
    n = d.shape[0]
    r = np.empty((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = tmin
    r[:, 4:7] = d
    r[:, 7] = tmax
    return r


def random_dirs(n, rng):
    return _unit(rng.normal(size=(n, 3)))


def surface_points(tris: np.ndarray, n: int, rng):
    idx = rng.integers(0, tris.shape[0], n)
    u = rng.random((n, 2))
    su = np.sqrt(u[:, 0])
    b = np.stack([1 - su, su * (1 - u[:, 1]), su * u[:, 1]], 1)
    t = tris[idx].astype(np.float64)
    return np.einsum("ni,nij->nj", b, t), idx


def edge_rays(tris: np.ndarray, n: int, rng, origin) -> np.ndarray:
    """Rays aimed exactly at vertices and edge midpoints (watertightness edge cases)."""
    idx = rng.integers(0, tris.shape[0], n)
    k = rng.integers(0, 6, n)
    t = tris[idx].astype(np.float64)
    targets = np.where(k[:, None] < 3, t[np.arange(n), k % 3],
                       0.5 * (t[np.arange(n), k % 3] + t[np.arange(n), (k + 1) % 3]))
    o = np.broadcast_to(np.asarray(origin, np.float64), targets.shape)
    return make_rays(o, _unit(targets - o), 0.0, np.finfo(np.float32).max)


# Ray categories stored with the fixtures: 0 camera, 1 interior, 2 leaving a surface point,
# 3 finite segment between surface points, 4 axis-aligned, 5 aimed at a vertex or edge midpoint.
CATEGORIES = ("camera", "interior", "surface", "segment", "axis", "edge")


def ray_set(scene_tris: np.ndarray, cam_scene: scenes.Scene, center, radius, rng):
    parts = [camera_rays(cam_scene, 48, 48, rng)]
    # interior rays with random directions
    o = center + (rng.random((2048, 3)) - 0.5) * radius
    parts.append(make_rays(o, random_dirs(2048, rng), 0.0, np.finfo(np.float32).max))
    # rays leaving surface points (origin exactly on a triangle, minT = 0)
    p, _ = surface_points(scene_tris, 2048, rng)
    parts.append(make_rays(p, random_dirs(2048, rng), 0.0, np.finfo(np.float32).max))
    # finite segments between surface points (shadow-ray shaped)
    p2, _ = surface_points(scene_tris, 2048, rng)
    p3, _ = surface_points(scene_tris, 2048, rng)
    seg = p3 - p2
    dist = np.linalg.norm(seg, axis=1)
    ok = dist > 1e-3
    parts.append(make_rays(p2[ok], seg[ok] / dist[ok, None], 0.0, (dist[ok] * 0.999)))
    # axis-aligned directions (zero direction components)
    axes = np.eye(3)[rng.integers(0, 3, 512)] * rng.choice([-1.0, 1.0], (512, 1))
    o = center + (rng.random((512, 3)) - 0.5) * radius
    parts.append(make_rays(o, axes, 0.0, np.finfo(np.float32).max))
    # vertices and edge midpoints
    parts.append(edge_rays(scene_tris, 1024, rng, cam_scene.cam_pos))
    cat = np.concatenate([np.full(p.shape[0], k, np.int32) for k, p in enumerate(parts)])
    return np.concatenate(parts).astype(np.float32), cat


def run_hits(tris: np.ndarray, ray_cat, name: str) -> None:
    rays, cat = ray_cat
    with tempfile.TemporaryDirectory() as tmp:
        tp, rp, op = (os.path.join(tmp, x) for x in ("t.f32", "r.f32", "o.bin"))
        np.ascontiguousarray(tris, np.float32).tofile(tp)
        np.ascontiguousarray(rays, np.float32).tofile(rp)
        subprocess.run([GOLDEN_TOOL, "hits", tp, rp, op], check=True)
        raw = np.fromfile(op, np.uint8).reshape(-1, 24)
    prim = raw[:, 0:4].copy().view(np.int32).ravel()
    tb = raw[:, 4:20].copy().view(np.float32).reshape(-1, 4)
    occ = raw[:, 20:24].copy().view(np.int32).ravel()
    np.savez_compressed(os.path.join(HERE, name), tris=tris.astype(np.float32), rays=rays,
                        category=cat, prim=prim, t=tb[:, 0], bary=tb[:, 1:4], occluded=occ)
    print(f"{name}: {tris.shape[0]} tris, {rays.shape[0]} rays, {np.mean(prim >= 0) * 100:.1f}% hit, "
          f"{np.mean(occ) * 100:.1f}% occluded")


def bsdf_cases(rng, n_per_type: int = 1500) -> np.ndarray:
    rows = []
    for typ in (0, 1, 2):
        n = n_per_type
        c = np.zeros((n, 19), np.float32)
        c[:, 0] = typ
        if typ == 0:
            c[:, 1:4] = rng.random((n, 3))
        elif typ == 1:
            c[:, 1] = rng.uniform(0.02, 0.8, n)
            c[:, 2:5] = rng.uniform(0.5, 1.0, (n, 3))
        else:
            c[:, 1] = rng.uniform(0.05, 0.6, n)
            c[:, 2] = 1.0
            c[:, 3] = rng.choice([1.5, 1.33, 2.4], n)
        N = random_dirs(n, rng)
        V = random_dirs(n, rng)
        L = random_dirs(n, rng)
        # bias a share of cases towards the same / opposite hemisphere of N
        flip = rng.random(n) < 0.35
        V[flip] = np.where((np.einsum("ij,ij->i", V, N) < 0)[flip, None], -V[flip], V[flip])
        c[:, 7:10] = N
        c[:, 10:13] = V
        c[:, 13:16] = L
        c[:, 16:19] = rng.random((n, 3))
        rows.append(c)
    return np.concatenate(rows)


def run_bsdf(cases: np.ndarray, name: str) -> None:
    with tempfile.TemporaryDirectory() as tmp:
        cp, op = os.path.join(tmp, "c.f32"), os.path.join(tmp, "o.f32")
        cases.tofile(cp)
        subprocess.run([GOLDEN_TOOL, "bsdf", cp, op], check=True)
        out = np.fromfile(op, np.float32).reshape(-1, 22)
    np.savez_compressed(os.path.join(HERE, name), cases=cases, out=out)
    print(f"{name}: {cases.shape[0]} cases, eval ok {out[:, 0].mean():.2f}, pdf ok {out[:, 4].mean():.2f}, "
          f"sample ok {out[:, 6].mean():.2f}")


def light_groups(num: int, rng, extent: float) -> list:
    """`num` area emitters of lognormal power (sigma 1) with random colour, size, position and
    orientation: mostly quads, every 7th a single triangle (the reference makes it a
    DiffuseSurfaceEmitter), every 11th a quad tessellated into 2 x 2 cells (8 triangles)."""
    groups = []
    for i in range(num):
        centre = rng.uniform(-extent, extent, 3)
        n = _unit(rng.normal(size=3))
        t = _unit(np.cross(n, [0.0, 1.0, 0.0] if abs(n[1]) < 0.9 else [1.0, 0.0, 0.0]))
        b = np.cross(n, t)
        su, sv = rng.uniform(0.05, 2.0, 2)
        radiance = rng.uniform(0.2, 1.0, 3) * np.exp(rng.normal(0.0, 1.0))
        if i % 7 == 3:
            tris = np.array([[centre, centre + su * t, centre + sv * b]])
        elif i % 11 == 5:
            cells = []
            for a in range(2):
                for c in range(2):
                    p0 = centre + (a * 0.5) * su * t + (c * 0.5) * sv * b
                    cells.append(scenes.quad(p0, p0 + 0.5 * su * t, p0 + 0.5 * su * t + 0.5 * sv * b, p0 + 0.5 * sv * b))
            tris = np.concatenate(cells)
        else:
            tris = scenes.quad(centre, centre + su * t, centre + su * t + sv * b, centre + sv * b)
        groups.append((np.asarray(tris, np.float32), radiance.astype(np.float32)))
    return groups


def run_lights(groups, rng, num_queries: int, extent: float, name: str) -> None:
    """Reference pick probabilities of every emitter and NEE densities of `num_queries` (receiving
    point, light triangle) pairs (oracle/_ref/ph_ref_golden lights)."""
    blob = [np.float32(len(groups))]
    for tris, rad in groups:
        blob.append(np.float32(tris.shape[0]))
        blob.extend(rad.astype(np.float32))
        blob.extend(tris.astype(np.float32).ravel())
    g_idx = rng.integers(0, len(groups), num_queries)
    t_idx = np.array([rng.integers(0, groups[g][0].shape[0]) for g in g_idx])
    targets = rng.uniform(-1.5 * extent, 1.5 * extent, (num_queries, 3)).astype(np.float32)
    q = np.zeros((num_queries, 6), np.float32)
    q[:, 0:3] = targets
    q[:, 3] = g_idx
    q[:, 4] = t_idx
    with tempfile.TemporaryDirectory() as tmp:
        gp, qp, op = (os.path.join(tmp, x) for x in ("g.f32", "q.f32", "o.f32"))
        np.asarray(blob, np.float32).tofile(gp)
        q.tofile(qp)
        subprocess.run([GOLDEN_TOOL, "lights", gp, qp, op], check=True)
        out = np.fromfile(op, np.float32)
    per_group = out[:2 * len(groups)].reshape(-1, 2)
    per_query = out[2 * len(groups):].reshape(-1, 6)
    first = np.cumsum([0] + [g[0].shape[0] for g in groups])
    np.savez_compressed(
        os.path.join(HERE, name),
        tris=np.concatenate([g[0] for g in groups]), group_first=first.astype(np.int64),
        radiance=np.stack([g[1] for g in groups]),
        flux=per_group[:, 0], pmf=per_group[:, 1],
        targets=targets, prim=(first[g_idx] + t_idx).astype(np.uint32),
        pdf_w=per_query[:, 0], emitter_pdf_w=per_query[:, 1], hit=per_query[:, 2] > 0, point=per_query[:, 3:6])
    print(f"{name}: {len(groups)} emitters, {num_queries} queries, {np.mean(per_query[:, 0] > 0) * 100:.0f}% "
          f"with a density, pmf {per_group[:, 1].min():.3g}..{per_group[:, 1].max():.3g}")


def c2_geometry():
    """The benchmarked 1M-triangle GGX scene's triangles (icosphere level 8, 1,310,726 triangles
    with the ground and the two lights) in scene order."""
    sc = scenes.ggx_sphere(level=8)
    return sc, np.ascontiguousarray(np.concatenate([g.tris for g in sc.groups]).astype(np.float32))


def c2_rays(tris: np.ndarray, sc: scenes.Scene, seed: int = 20261205):
    """32,768-odd rays over the benchmarked scene, in the categories of ray_set (camera rays through
    a 64 x 64 jittered grid, interior, leaving surfaces, segments between surface points,
    axis-aligned, aimed at vertices and edge midpoints), regenerated from `seed`."""
    rng = np.random.default_rng(seed)
    center, radius = np.array([0.0, 1.0, 0.0]), 3.0
    parts = [camera_rays(sc, 64, 64, rng)]
    o = center + (rng.random((8192, 3)) - 0.5) * radius
    parts.append(make_rays(o, random_dirs(8192, rng), 0.0, np.finfo(np.float32).max))
    p, _ = surface_points(tris, 8192, rng)
    parts.append(make_rays(p, random_dirs(8192, rng), 0.0, np.finfo(np.float32).max))
    p2, _ = surface_points(tris, 8192, rng)
    p3, _ = surface_points(tris, 8192, rng)
    seg = p3 - p2
    dist = np.linalg.norm(seg, axis=1)
    ok = dist > 1e-3
    parts.append(make_rays(p2[ok], seg[ok] / dist[ok, None], 0.0, (dist[ok] * 0.999)))
    axes = np.eye(3)[rng.integers(0, 3, 2048)] * rng.choice([-1.0, 1.0], (2048, 1))
    o = center + (rng.random((2048, 3)) - 0.5) * radius
    parts.append(make_rays(o, axes, 0.0, np.finfo(np.float32).max))
    parts.append(edge_rays(tris, 2048, rng, sc.cam_pos))
    cat = np.concatenate([np.full(q.shape[0], k, np.int32) for k, q in enumerate(parts)])
    return np.ascontiguousarray(np.concatenate(parts).astype(np.float32)), cat


def sha256(a: np.ndarray) -> str:
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_c2_hits() -> None:
    """c2_hits.npz: the reference's closest hits and occlusion on the benchmarked scene. The
    triangles and rays are regenerated by the test (c2_geometry, c2_rays); their SHA-256 digests
    are stored so that a test on regenerated inputs knows they are the same bits."""
    sc, tris = c2_geometry()
    rays, cat = c2_rays(tris, sc)
    with tempfile.TemporaryDirectory() as tmp:
        tp, rp, op = (os.path.join(tmp, x) for x in ("t.f32", "r.f32", "o.bin"))
        tris.tofile(tp)
        rays.tofile(rp)
        subprocess.run([GOLDEN_TOOL, "hits", tp, rp, op], check=True)
        raw = np.fromfile(op, np.uint8).reshape(-1, 24)
    prim = raw[:, 0:4].copy().view(np.int32).ravel()
    tb = raw[:, 4:20].copy().view(np.float32).reshape(-1, 4)
    occ = raw[:, 20:24].copy().view(np.int32).ravel()
    np.savez_compressed(os.path.join(HERE, "c2_hits.npz"), tris_sha256=sha256(tris), rays_sha256=sha256(rays),
                        num_tris=tris.shape[0], category=cat, prim=prim, t=tb[:, 0], occluded=occ.astype(np.int8))
    print(f"c2_hits.npz: {tris.shape[0]} tris, {rays.shape[0]} rays, {np.mean(prim >= 0) * 100:.1f}% hit, "
          f"{np.mean(occ) * 100:.1f}% occluded")


def main() -> None:
    """Writes every fixture, or only the parts named on the command line (hits, bsdf, lights, c2)."""
    if not os.path.exists(GOLDEN_TOOL):
        raise SystemExit(f"{GOLDEN_TOOL} missing: run `make -f oracle/Makefile.ref REF=<reference sources> -j8` first")
    parts = set(sys.argv[1:]) or {"hits", "bsdf", "lights", "c2"}
    rng = np.random.default_rng(20261203)

    cb = scenes.cornell()
    cb_tris = np.concatenate([g.tris for g in cb.groups])
    cb_rays = ray_set(cb_tris, cb, np.array([277.5, 277.5, 277.5]), 500.0, rng)
    sp = scenes.ggx_sphere(level=4, with_env=False)
    sp_tris = np.concatenate([g.tris for g in sp.groups])
    sp_rays = ray_set(sp_tris, sp, np.array([0.0, 1.0, 0.0]), 3.0, rng)
    if "hits" in parts:
        run_hits(cb_tris, cb_rays, "hits_cornell.npz")
        run_hits(sp_tris, sp_rays, "hits_sphere.npz")
    cases = bsdf_cases(rng)
    if "bsdf" in parts:
        run_bsdf(cases, "bsdf_cases.npz")

    if "lights" in parts:
        lrng = np.random.default_rng(20261204)
        for count, queries, extent in ((3, 600, 3.0), (100, 1500, 10.0), (10_000, 2400, 60.0)):
            run_lights(light_groups(count, lrng, extent), lrng, queries, extent, f"lights_{count}.npz")

    if "c2" in parts:
        run_c2_hits()


if __name__ == "__main__":
    main()
