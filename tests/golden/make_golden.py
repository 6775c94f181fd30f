"""Generates the golden fixtures of the parity tests by running the reference's own code.

Run in the build container, where the reference sources exist and the oracle has been built
(``make -f oracle/Makefile.ref -j8``):

    python tests/golden/make_golden.py

It writes, next to this script:
  hits_cornell.npz, hits_sphere.npz   rays + closest-hit primitive/t/barycentrics + occlusion,
                                      computed by the reference's TBinaryBvhIntersector over
                                      PTriangles (oracle/_ref/ph_ref_golden hits)
  bsdf_cases.npz                      BSDF eval/pdf/sample answers of LambertianReflector,
                                      OpaqueMicrofacet and TranslucentMicrofacet
                                      (oracle/_ref/ph_ref_golden bsdf)
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


def main() -> None:
    if not os.path.exists(GOLDEN_TOOL):
        raise SystemExit(f"{GOLDEN_TOOL} missing: run `make -f oracle/Makefile.ref -j8` first")
    rng = np.random.default_rng(20261203)

    cb = scenes.cornell()
    cb_tris = np.concatenate([g.tris for g in cb.groups])
    run_hits(cb_tris, ray_set(cb_tris, cb, np.array([277.5, 277.5, 277.5]), 500.0, rng), "hits_cornell.npz")

    sp = scenes.ggx_sphere(level=4, with_env=False)
    sp_tris = np.concatenate([g.tris for g in sp.groups])
    run_hits(sp_tris, ray_set(sp_tris, sp, np.array([0.0, 1.0, 0.0]), 3.0, rng), "hits_sphere.npz")

    run_bsdf(bsdf_cases(rng), "bsdf_cases.npz")


if __name__ == "__main__":
    main()
