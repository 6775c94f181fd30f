"""The GPU BVH builder (Morton-ordered radix tree collapsed to the 8-wide layout).

A tree never changes the answer of a closest-hit or occlusion query, only its cost, so the GPU-built
tree is held to the same bar as the host SAH tree against the reference's own answers
(tests/golden/hits_*.npz), and the two trees must agree with each other ray by ray. The exported
tree is also checked structurally: every triangle sits in exactly one leaf, and every triangle of a
subtree lies inside the quantised box the subtree's parent decodes for it (decoded in FP32 exactly
as the traversal does).
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from test_trace_parity import ulp_diff

import scenes


def _decode_boxes(node):
    """[8] slot boxes (lo [8,3], hi [8,3]) and per-slot meta of one wide node (uint32[20])."""
    p = node[0:3].view(np.float32)
    ex = [int((node[3] >> (8 * a)) & 0xFF) - 127 for a in range(3)]
    scale = np.array([np.ldexp(np.float32(1.0), e) for e in ex], np.float32)
    meta = [(int(node[6 + s // 4]) >> (8 * (s % 4))) & 0xFF for s in range(8)]
    lo = np.zeros((8, 3), np.float32)
    hi = np.zeros((8, 3), np.float32)
    for a in range(3):
        for s in range(8):
            ql = (int(node[8 + 2 * a + s // 4]) >> (8 * (s % 4))) & 0xFF
            qh = (int(node[14 + 2 * a + s // 4]) >> (8 * (s % 4))) & 0xFF
            lo[s, a] = np.float32(p[a] + np.float32(ql) * scale[a])
            hi[s, a] = np.float32(p[a] + np.float32(qh) * scale[a])
    return lo, hi, meta


def _check_tree(nodes, tris, num_prims):
    """Every triangle in exactly one leaf; every triangle of a subtree inside the box its parent's
    slot decodes for that subtree."""
    import sys

    assert sorted(tris["prim"].tolist()) == list(range(num_prims))
    sys.setrecursionlimit(10000)
    seen = np.zeros(len(tris), bool)

    def subtree(ni):
        node = nodes[ni]
        lo, hi, meta = _decode_boxes(node)
        imask = int(node[3] >> 24)
        child_base, tri_base = int(node[4]), int(node[5])
        verts = []
        for s in range(8):
            m = meta[s]
            if m == 0:
                continue
            if (imask >> s) & 1:
                rank = bin(imask & ((1 << s) - 1)).count("1")
                v = subtree(child_base + rank)
            else:
                unary, off = m >> 5, m & 31
                idx = [tri_base + off + b for b in range(3) if (unary >> b) & 1]
                assert not seen[idx].any()
                seen[idx] = True
                t = tris[idx]
                v = np.concatenate([t["v0"], t["v1"], t["v2"]])
            ok = np.all((v >= lo[s]) & (v <= hi[s]), axis=1) | ~np.all(np.isfinite(v), axis=1)
            assert ok.all(), (ni, s)
            verts.append(v)
        return np.concatenate(verts)

    subtree(0)
    assert seen.all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["hits_cornell.npz", "hits_sphere.npz"])
def test_gpu_built_tree_gives_the_reference_hits(gpu_lib, name):
    import photon_gpu

    d = dict(np.load(os.path.join(GOLDEN, name)))
    mo = float(np.abs(d["rays"][:, :3]).max())
    with photon_gpu.Geometry(d["tris"], max_origin_abs=mo, builder="gpu") as g:
        prim, t, bary = g.closest(d["rays"])
        occ = g.occluded(d["rays"])
        nodes, tris = g.export()
    _check_tree(nodes, tris, d["tris"].shape[0])
    hit_ref = d["prim"] >= 0
    assert np.array_equal(prim >= 0, hit_ref)
    same = (prim == d["prim"]) & hit_ref
    near_tie = hit_ref & ~same & (ulp_diff(t, d["t"]) <= 2)
    assert np.all(same | near_tie | ~hit_ref)
    assert near_tie.sum() <= 0.06 * hit_ref.sum()
    assert np.array_equal(t[same].view(np.uint32), d["t"][same].view(np.uint32))
    assert np.array_equal(occ, d["occluded"])
    # and ray by ray the same as the host SAH tree (up to the same near-ties)
    with photon_gpu.Geometry(d["tris"], max_origin_abs=mo, builder="sah") as g2:
        prim2, t2, _ = g2.closest(d["rays"])
    agree = (prim == prim2) | (ulp_diff(t, t2) <= 2)
    assert agree.all()


@pytest.mark.gpu
def test_gpu_build_of_degenerate_inputs(gpu_lib):
    import photon_gpu

    rng = np.random.default_rng(4)
    one = np.array([[[0, 0, 1], [1, 0, 1], [0, 1, 1]]], np.float32)
    copies = np.repeat(one, 1000, axis=0)                       # identical centroids
    mixed = np.concatenate([copies, rng.random((3000, 3, 3)).astype(np.float32)])
    for tris in (one, one[[0, 0]], copies, mixed):
        rays = np.zeros((256, 8), np.float32)
        rays[:, 0:2] = rng.random((256, 2)) * 0.6
        rays[:, 2] = -1.0
        rays[:, 6] = 1.0
        rays[:, 7] = 1e30
        with photon_gpu.Geometry(tris, builder="gpu") as g:
            prim, t, _ = g.closest(rays)
            nodes, leaf = g.export()
            stats = g.stats()
        with photon_gpu.Geometry(tris, builder="sah") as h:
            prim_h, t_h, _ = h.closest(rays)
        _check_tree(nodes, leaf, tris.shape[0])
        assert stats["max_depth"] < 64
        assert np.array_equal(prim >= 0, prim_h >= 0)
        assert np.array_equal(t.view(np.uint32), t_h.view(np.uint32))


@pytest.mark.gpu
def test_render_with_gpu_built_tree_matches_reference(gpu_lib):
    import photon_gpu

    d = np.load(os.path.join(GOLDEN, "images.npz"))
    ref = d["ggx_sphere_env_bneept"]
    scene = scenes.ggx_sphere(level=3, width=64, height=64, spp=4096, max_bounces=10)
    with photon_gpu.RenderScene(scene, builder="gpu") as rs:
        rs.render(4096, max_bounces=10, seed=1)
        img = rs.film()[0]
    block = lambda a: a.reshape(16, 4, 16, 4, 3).mean(axis=(1, 3)).astype(np.float64)
    err = float(np.mean((block(img) - block(ref)) ** 2 / (block(ref) ** 2 + 1e-2)))
    means = img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1))
    assert err <= 1e-3 and np.all(np.abs(means - 1) < 0.01), (err, means)


@pytest.mark.gpu
@pytest.mark.parametrize("builder", ["sah", "gpu"])
def test_city_traversal_stays_within_the_stack(gpu_lib, builder):
    """The many-light city at full size (21,599,374 triangles, 10,000 lights): both builders keep
    the 8-wide tree shallower than the 64-entry traversal stack (the builders refuse deeper trees),
    and a render of the scene, whose traversal kernels raise a device flag on any stack overflow,
    completes (an overflow ends the render with PG_ERR_STACK_OVERFLOW)."""
    import photon_gpu

    sc = scenes.city(96, 54, 4, 12)
    with photon_gpu.RenderScene(sc, builder=builder) as rs:
        rs.render(4, max_bounces=12, seed=3)
        rgb = rs.film(with_sums=False)[0]
    assert np.all(np.isfinite(rgb)) and rgb.mean() > 0
    tris = np.concatenate([g.tris for g in sc.groups])
    with photon_gpu.Geometry(tris, builder=builder) as g:
        depth = g.stats()["max_depth"]
    print(f"city ({builder}): {tris.shape[0]} triangles, wide-tree depth {depth}")
    assert depth < 64
