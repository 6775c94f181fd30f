"""ctypes binding of the oracle's CPU restatement (oracle/_build/libph_port.so).

Test infrastructure only: the parity tests use it as a checker, bench.py's CPU baseline may run
its CLI when the reference build is missing. Build with ``make -f oracle/Makefile.port``.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(_HERE), "_build", "libph_port.so")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} missing: run `make -f oracle/Makefile.port`")
        _lib = ctypes.CDLL(LIB)
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def trace(tris, rays):
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = r.shape[0]
    prim = np.empty(n, np.int32)
    th = np.empty(n, np.float32)
    bary = np.empty((n, 3), np.float32)
    occ = np.empty(n, np.int32)
    load().port_trace(_p(t, ctypes.c_float), ctypes.c_uint32(t.shape[0]), _p(r, ctypes.c_float),
                      ctypes.c_uint32(n), _p(prim, ctypes.c_int32), _p(th, ctypes.c_float),
                      _p(bary, ctypes.c_float), _p(occ, ctypes.c_int32))
    return prim, th, bary, occ


def bsdf(cases, normals):
    c = np.ascontiguousarray(cases, np.float32).reshape(-1, 19)
    nrm = np.ascontiguousarray(normals, np.float32).reshape(-1, 6)
    out = np.empty((c.shape[0], 16), np.float32)
    load().port_bsdf(_p(c, ctypes.c_float), _p(nrm, ctypes.c_float), ctypes.c_uint32(c.shape[0]),
                     _p(out, ctypes.c_float))
    return out


FILTERS = {"box": 0, "gaussian": 1, "mn": 2, "bh": 3}


def render(flat_scene, spp, max_bounces, estimator=0, threads=None, seed=1, sample_filter=None):
    """Renders the flat scene arrays of photon_gpu.flatten_scene; returns float32 [H, W, 3].

    Without `sample_filter` every pixel averages its own samples (box filter); with one of
    FILTERS the samples are splatted through that filter into an (R, G, B, W) film."""
    tris, tri_mat, tri_em, mats, ems, cam = flat_scene
    w, h = int(cam[10]), int(cam[11])
    threads = threads or (os.cpu_count() or 1)
    ems = np.ascontiguousarray(ems, np.float32)
    args = [
        _p(np.ascontiguousarray(tris, np.float32), ctypes.c_float), _p(np.ascontiguousarray(tri_mat, np.uint32), ctypes.c_uint32),
        _p(np.ascontiguousarray(tri_em, np.uint32), ctypes.c_uint32), ctypes.c_uint32(tris.shape[0]),
        _p(np.ascontiguousarray(mats, np.float32), ctypes.c_float), ctypes.c_uint32(mats.shape[0]),
        _p(ems, ctypes.c_float) if ems.size else None, ctypes.c_uint32(ems.shape[0]),
        _p(np.ascontiguousarray(cam, np.float32), ctypes.c_float), ctypes.c_uint32(spp),
        ctypes.c_uint32(max_bounces), ctypes.c_uint32(estimator), ctypes.c_uint32(threads),
        ctypes.c_uint64(seed)]
    if sample_filter is not None:
        sums = np.zeros((h, w, 4), np.float64)
        status = load().port_render_filtered(*args, ctypes.c_uint32(FILTERS[sample_filter]), _p(sums, ctypes.c_double))
        if status != 0:
            raise RuntimeError("port_render_filtered failed")
        wsum = sums[..., 3:4]
        return (sums[..., :3] / np.where(wsum != 0, wsum, 1.0) * (wsum != 0)).astype(np.float32)
    sums = np.zeros((h, w, 3), np.float64)
    status = load().port_render(*args, _p(sums, ctypes.c_double))
    if status != 0:
        raise RuntimeError("port_render failed")
    return (sums / spp).astype(np.float32)


def rotation_matrix(axis, degrees):
    """Row-major rotation by `degrees` about `axis` (right-handed), as an actor's rotate() sets it."""
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    t = np.radians(degrees)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(t) * k + (1 - np.cos(t)) * (k @ k)


def set_environment(image=None, rotation=None, center=(0.0, 0.0, 0.0), exact=False):
    """The dome of the following renders: `image` [H, W, 3] with row 0 at the top (as written to a
    PFM by scenes.write_pfm), or None for the scene's constant environment; `rotation` (axis,
    degrees) of the dome; `exact` for the true sample densities instead of the reference's."""
    rot = np.ascontiguousarray(rotation_matrix(*rotation) if rotation else np.eye(3), np.float32)
    c = np.ascontiguousarray(center, np.float32)
    if image is None:
        load().port_set_environment(None, 0, 0, _p(rot, ctypes.c_float), _p(c, ctypes.c_float), int(exact))
        return
    img = np.ascontiguousarray(np.asarray(image, np.float32)[::-1])   # row 0 = bottom
    load().port_set_environment(_p(img, ctypes.c_float), img.shape[1], img.shape[0], _p(rot, ctypes.c_float),
                                _p(c, ctypes.c_float), int(exact))


def write_scene_bin(path, flat_scene, spp, estimator=0):
    """The scene file ph_port_render reads (see oracle/port/ph_port.cpp)."""
    tris, tri_mat, tri_em, mats, ems, cam = flat_scene
    with open(path, "wb") as f:
        f.write(b"PHPT")
        np.array([1, int(cam[10]), int(cam[11]), spp, estimator], np.uint32).tofile(f)
        np.asarray(cam, np.float32).tofile(f)
        np.array([tris.shape[0], mats.shape[0], ems.shape[0]], np.uint32).tofile(f)
        np.ascontiguousarray(tris, np.float32).tofile(f)
        np.ascontiguousarray(tri_mat, np.uint32).tofile(f)
        np.ascontiguousarray(tri_em, np.uint32).tofile(f)
        np.ascontiguousarray(mats, np.float32).tofile(f)
        np.ascontiguousarray(ems, np.float32).tofile(f)
