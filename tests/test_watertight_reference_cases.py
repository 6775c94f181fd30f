"""The reference's own known answers for the watertight ray-triangle test.

Engine/EngineTest/Source/Math/Geometry/TWatertightTriangle_test.cpp holds two tests:

* IsDegenerate (:11-59): a right triangle and a large, skewed triangle with coordinates up to 9e4
  are proper triangles; triangles with an infinite, a quiet-NaN or a signalling-NaN coordinate
  are degenerate.
* TolerateNonFiniteVertices (:61-78): the triangle (0,0,0), (1,1,0), (1,-1,+inf) is not hit by
  the segment from (0.1, 0, -1) along (0.1, 0, 1) over [0, FLT_MAX) (TLineSegment.ipp:14-20),
  although it would be if +inf were treated like an ordinary value >= 0.

Here each triangle is a scene of its own, traced by a ray through the interior its finite
vertices span: the proper triangles are hit at the t their plane gives, and the degenerate ones
are never hit, also when they share a tree with proper triangles. The CPU restatement
(oracle/port) must give these answers, and so must the GPU traversal through the C ABI, with
the tree from either builder (host SAH and GPU PLOC). The GPU's t must equal the restatement's
bit for bit (both compute the reference's FP32 operation order) and lie within two FP32 spacings
of the largest coordinate involved (vertices and ray origin) of the FP64 plane intersection.
"""

import numpy as np
import pytest

INF = np.float32(np.inf)
QNAN = np.float32(np.nan)
SNAN = np.array([0x7FA00000], np.uint32).view(np.float32)[0]   # exponent all ones, quiet bit clear
FLT_MAX = np.finfo(np.float32).max


def _ray(origin, direction, tmin=0.0, tmax=FLT_MAX):
    return np.array([*origin, tmin, *direction, tmax], np.float32)


# (name, triangle [3, 3], ray [8], hit expected)
CASES = [
    ("right triangle", [[0, 0, 0], [1, 0, 0], [0, 1, 0]], _ray((0.25, 0.25, -1.0), (0.0, 0.0, 1.0)), True),
    ("large skewed triangle",
     [[0, 0, 0], [10000.0, 50000.0, 90000.0], [70000.0, 30000.0, -10000.0]], None, True),
    ("infinite vertex", [[0, 0, 0], [1, 0, 0], [0, 1, INF]], _ray((0.25, 0.25, -1.0), (0.0, 0.0, 1.0)), False),
    ("quiet NaN vertex", [[0, 0, 0], [1, 0, QNAN], [0, 1, 0]], _ray((0.25, 0.25, -1.0), (0.0, 0.0, 1.0)), False),
    ("signalling NaN vertex", [[0, 0, SNAN], [1, 0, 0], [0, 1, 0]], _ray((0.25, 0.25, -1.0), (0.0, 0.0, 1.0)), False),
    ("non-finite vertex tolerated", [[0, 0, 0], [1, 1, 0], [1, -1, INF]], _ray((0.1, 0.0, -1.0), (0.1, 0.0, 1.0)), False),
]


def _large_triangle_ray(tri):
    """A ray from 100 units off the triangle's centroid, along its normal, back towards it."""
    v = tri.astype(np.float64)
    c = v.mean(0)
    n = np.cross(v[1] - v[0], v[2] - v[0])
    n /= np.linalg.norm(n)
    return _ray(tuple(c + 100.0 * n), tuple(-n))


def _cases():
    out = []
    for name, tri, ray, hit in CASES:
        tri = np.array(tri, np.float32)
        if ray is None:
            ray = _large_triangle_ray(tri)
        out.append((name, tri, ray, hit))
    return out


def _plane_t(tri, ray):
    """t of the ray's crossing with the triangle's plane, in FP64."""
    v = tri.astype(np.float64)
    o, d = ray[:3].astype(np.float64), ray[4:7].astype(np.float64)
    n = np.cross(v[1] - v[0], v[2] - v[0])
    return float(np.dot(v[0] - o, n) / np.dot(d, n))


def _combined():
    """All six triangles in one scene (the proper ones moved apart) with all six rays."""
    tris, rays, expect = [], [], []
    for k, (_, tri, ray, hit) in enumerate(_cases()):
        shift = np.float32(1000.0 * (k + 1))   # proper triangles away from the other rays
        tris.append(tri + np.array([shift, 0, 0], np.float32) if hit else tri)
        r = ray.copy()
        if hit:
            r[0] += shift
        rays.append(r)
        expect.append(k if hit else -1)
    return np.stack(tris), np.stack(rays), np.array(expect)


def _check(name, tri, ray, hit, prim, t):
    if hit:
        assert prim == 0, f"{name}: expected a hit"
        scale = max(float(np.abs(tri).max()), float(np.abs(ray[:3]).max()))
        assert abs(float(t) - _plane_t(tri, ray)) <= 2.0 * float(np.spacing(np.float32(scale))), name
    else:
        assert prim == -1, f"{name}: a triangle with a non-finite vertex was hit (t = {t})"


def _port():
    import os
    import subprocess

    from conftest import ROOT
    from oracle.port import port as p

    if not os.path.exists(p.LIB):
        subprocess.run(["make", "-f", "oracle/Makefile.port"], cwd=ROOT, check=True, stdout=subprocess.DEVNULL)
    p.load()
    return p


@pytest.mark.parametrize("case", range(len(CASES)), ids=[c[0] for c in CASES])
def test_port_reference_cases(case):
    p = _port()
    name, tri, ray, hit = _cases()[case]
    with np.errstate(invalid="ignore"):
        prim, t, _, occ = p.trace(tri[None], ray[None])
    _check(name, tri, ray, hit, int(prim[0]), t[0])
    assert bool(occ[0]) == hit


def test_port_reference_cases_in_one_tree():
    p = _port()
    tris, rays, expect = _combined()
    prim, _, _, occ = p.trace(tris, rays)
    assert np.array_equal(prim, expect)
    assert np.array_equal(occ.astype(bool), expect >= 0)


@pytest.mark.gpu
@pytest.mark.parametrize("builder", ["sah", "gpu"])
def test_gpu_reference_cases(gpu_lib, builder):
    import photon_gpu

    p = _port()
    for name, tri, ray, hit in _cases():
        with photon_gpu.Geometry(tri[None], max_origin_abs=float(np.abs(ray[:3]).max()), builder=builder) as g:
            prim, t, _ = g.closest(ray[None])
            occ = g.occluded(ray[None])
        _check(name, tri, ray, hit, int(prim[0]), t[0])
        assert bool(occ[0]) == hit, name
        if hit:
            _, t_port, _, _ = p.trace(tri[None], ray[None])
            assert t.view(np.uint32)[0] == t_port.view(np.uint32)[0], f"{name}: t differs from the restatement"

    tris, rays, expect = _combined()
    with photon_gpu.Geometry(tris, max_origin_abs=float(np.abs(rays[:, :3]).max()), builder=builder) as g:
        prim, _, _ = g.closest(rays)
        occ = g.occluded(rays)
    assert np.array_equal(prim, expect)
    assert np.array_equal(np.asarray(occ).astype(bool), expect >= 0)
