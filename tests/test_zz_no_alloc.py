"""pgpu_trace_closest_noalloc: the closest-hit query that allocates nothing.

Called through the C ABI (ctypes on libphoton_gpu.so) and compared with pgpu_trace_closest on the
same geometry and rays. Both run the same traversal and resolve kernels, so the tolerance is
exact equality of prim, t and barycentrics. Two calls in a row must both agree (the static scratch
is reused, nothing in it is assumed to start at zero). Sizes above the scratch capacity are
rejected with PG_ERR_INVALID_ARGUMENT. The file is named to be collected last, so the suite also
exercises the entry point after every other GPU test has run in the same process.
"""

import ctypes
import os

import numpy as np
import pytest

from conftest import GOLDEN

MAX_RAYS = 1 << 16
PG_ERR_INVALID_ARGUMENT = 1


def _noalloc(lib, gid, rays):
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = r.shape[0]
    prim = np.full(n, -7, np.int32)
    t = np.full(n, np.nan, np.float32)
    bary = np.full((n, 3), np.nan, np.float32)
    status = lib.pgpu_trace_closest_noalloc(
        gid, r.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n,
        prim.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
        t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
        bary.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return status, prim, t, bary


def _rays_for(d, n, seed):
    """n rays drawn (with jitter) from the fixture's rays."""
    rng = np.random.default_rng(seed)
    base = d["rays"][rng.integers(0, d["rays"].shape[0], n)].copy()
    base[:, 0:3] += rng.normal(0.0, 1e-3, (n, 3)).astype(np.float32)
    return base


@pytest.mark.gpu
@pytest.mark.parametrize("fixture", ["hits_sphere.npz", "hits_cornell.npz"])
def test_noalloc_matches_allocating_entry_point(gpu_lib, fixture):
    import photon_gpu

    d = np.load(os.path.join(GOLDEN, fixture))
    with photon_gpu.Geometry(d["tris"], max_origin_abs=float(np.abs(d["rays"][:, :3]).max()) + 1.0) as g:
        for rays in (d["rays"], _rays_for(d, MAX_RAYS, 11)):
            prim, t, bary = g.closest(rays)
            for _ in range(2):   # two calls in a row reuse the same scratch
                status, p2, t2, b2 = _noalloc(gpu_lib, g.id, rays)
                assert status == 0, gpu_lib.pgpu_last_error()
                assert np.array_equal(p2, prim)
                assert np.array_equal(t2.view(np.uint32), t.view(np.uint32))
                assert np.array_equal(b2.view(np.uint32), bary.view(np.uint32))


@pytest.mark.gpu
def test_noalloc_rejects_oversized_batches_and_accepts_empty(gpu_lib):
    import photon_gpu

    d = np.load(os.path.join(GOLDEN, "hits_cornell.npz"))
    with photon_gpu.Geometry(d["tris"]) as g:
        status, *_ = _noalloc(gpu_lib, g.id, np.zeros((0, 8), np.float32))
        assert status == 0
        status, prim, _, _ = _noalloc(gpu_lib, g.id, _rays_for(d, MAX_RAYS + 1, 3))
        assert status == PG_ERR_INVALID_ARGUMENT
        assert b"exceed" in gpu_lib.pgpu_last_error()
        assert np.all(prim == -7)   # rejected before any work
        # still usable afterwards
        status, prim, _, _ = _noalloc(gpu_lib, g.id, d["rays"][:64])
        assert status == 0 and np.array_equal(prim, g.closest(d["rays"][:64])[0])
