"""ctypes binding of libphoton_gpu.so: the low-level C ABI (include/photon_gpu.h) and the Photon C
API (include/ph_c_core.h) exported by the same library.

The library is built in-tree (``make -C photon-v2_b200``). Loading fails loudly when it is missing:
there is no CPU fallback for any entry point.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libphoton_gpu.so")

_lib: Optional[ctypes.CDLL] = None

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_dblp = ctypes.POINTER(ctypes.c_double)

# (name, restype, argtypes) of every exported entry point.
PGPU_SIGNATURES = [
    ("pgpu_last_error", ctypes.c_char_p, []),
    ("pgpu_device_count", ctypes.c_int, []),
    ("pgpu_geometry_create", ctypes.c_int, [_f32p, ctypes.c_uint64, ctypes.c_float, _u64p]),
    ("pgpu_geometry_create_ex", ctypes.c_int, [_f32p, ctypes.c_uint64, ctypes.c_float, ctypes.c_uint32, _u64p]),
    ("pgpu_geometry_export", ctypes.c_int, [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, _u64p, _u64p]),
    ("pgpu_geometry_destroy", ctypes.c_int, [ctypes.c_uint64]),
    ("pgpu_geometry_stats", ctypes.c_int, [ctypes.c_uint64, _u64p, _u64p, _i32p, _dblp]),
    ("pgpu_trace_closest", ctypes.c_int, [ctypes.c_uint64, _f32p, ctypes.c_uint64, _i32p, _f32p, _f32p]),
    ("pgpu_trace_any", ctypes.c_int, [ctypes.c_uint64, _f32p, ctypes.c_uint64, _i32p]),
    ("pgpu_trace_closest_noalloc", ctypes.c_int,
     [ctypes.c_uint64, _f32p, ctypes.c_uint64, _i32p, _f32p, _f32p]),
    ("pgpu_trace_closest_device", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, _f32p]),
    ("pgpu_trace_any_device", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, _f32p]),
    ("pgpu_trace_counts", ctypes.c_int,
     [ctypes.c_uint64, _f32p, ctypes.c_uint64, ctypes.c_int, _dblp, _dblp]),
    ("pgpu_bsdf_eval", ctypes.c_int, [_f32p, _f32p, ctypes.c_uint64, _f32p]),
    ("pgpu_film_splat", ctypes.c_int,
     [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _f32p, ctypes.c_uint64, _dblp]),
    ("pgpu_guide_forward", ctypes.c_int, [_f32p, _f32p, ctypes.c_uint64, _f32p]),
    ("pgpu_guide_mixture", ctypes.c_int, [_f32p, _f32p, ctypes.c_uint64, _f32p]),
    ("pgpu_guide_gradients", ctypes.c_int, [_f32p, _f32p, _f32p, _f32p, ctypes.c_uint64, _f32p, _f32p]),
    ("pgpu_guide_gradients_ex", ctypes.c_int,
     [_f32p, _f32p, _f32p, _f32p, ctypes.c_uint64, ctypes.c_uint32, _f32p, _f32p]),
    ("pgpu_guide_train", ctypes.c_int,
     [_f32p, _f32p, _f32p, _f32p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, _f32p]),
    ("pgpu_scene_create", ctypes.c_int,
     [_f32p, _u32p, _u32p, ctypes.c_uint64, _f32p, ctypes.c_uint32, _f32p, ctypes.c_uint32, _f32p, _u64p]),
    ("pgpu_scene_create_ex", ctypes.c_int,
     [_f32p, _u32p, _u32p, ctypes.c_uint64, _f32p, ctypes.c_uint32, _f32p, ctypes.c_uint32, _f32p, ctypes.c_uint32,
      _u64p]),
    ("pgpu_scene_destroy", ctypes.c_int, [ctypes.c_uint64]),
    ("pgpu_scene_render", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
      _f32p, _u64p, _u64p]),
    ("pgpu_scene_film", ctypes.c_int, [ctypes.c_uint64, _f32p, _dblp, _u64p]),
    ("pgpu_scene_clear", ctypes.c_int, [ctypes.c_uint64]),
    ("pgpu_scene_set_filter", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32]),
    ("pgpu_scene_set_dome_pdf", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32]),
    ("pgpu_scene_launches", ctypes.c_int, [ctypes.c_uint64, _u64p]),
    ("pgpu_scene_light_pmf", ctypes.c_int, [ctypes.c_uint64, _f32p, _dblp, _u32p]),
    ("pgpu_scene_autotune", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, _u32p,
      _f32p]),
    ("pgpu_scene_set_launch", ctypes.c_int, [ctypes.c_uint64, _u32p]),
    ("pgpu_scene_get_launch", ctypes.c_int, [ctypes.c_uint64, _u32p]),
    ("pgpu_scene_light_pdf", ctypes.c_int, [ctypes.c_uint64, _f32p, _u32p, ctypes.c_uint64, _f32p]),
    ("pgpu_scenes_render", ctypes.c_int,
     [_u64p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, _f32p]),
    ("pgpu_scenes_render_wavefront", ctypes.c_int,
     [_u64p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _f32p]),
    ("pgpu_scenes_autotune_wavefront", ctypes.c_int,
     [_u64p, ctypes.c_uint32, _u32p, ctypes.c_uint32, ctypes.c_uint32, _u32p, _f32p]),
    ("pgpu_scene_count", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _u64p]),
    ("pgpu_scene_profile", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _dblp]),
    ("pgpu_scene_set_guiding", ctypes.c_int,
     [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_uint32]),
    ("pgpu_scene_set_guiding_depth", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32]),
    ("pgpu_scene_guide_reset", ctypes.c_int, [ctypes.c_uint64]),
    ("pgpu_scene_guide_info", ctypes.c_int, [ctypes.c_uint64, _f32p, _u64p, _dblp, _f32p]),
    ("pgpu_sdl_cook", ctypes.c_int,
     [ctypes.c_char_p, ctypes.c_char_p, _u64p, _u32p, _u32p, _u32p, _f32p, _u32p, _u32p, _f32p, _f32p]),
]


class PhotonGpuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the library (once) and declares all signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `make -C photon-v2_b200` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, res, args in PGPU_SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _declare_ph_api(lib)
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != 0:
        msg = load().pgpu_last_error().decode(errors="replace")
        raise PhotonGpuError(status, msg)


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def device_count() -> int:
    return int(load().pgpu_device_count())


BUILDERS = {"sah": 0, "gpu": 1}
# 48-byte leaf triangle: v0 xyz, original index, v1 xyz, material, v2 xyz, emitter + 1
LEAF_TRI_DTYPE = np.dtype([("v0", np.float32, 3), ("prim", np.uint32), ("v1", np.float32, 3),
                           ("material", np.uint32), ("v2", np.float32, 3), ("emitter", np.uint32)])


class Geometry:
    """Triangles [N, 3, 3] with their 8-wide BVH resident on the GPU."""

    def __init__(self, tris: np.ndarray, max_origin_abs: float = 0.0, builder: str = "sah"):
        """builder: "sah" (host binned SAH) or "gpu" (Morton-ordered radix tree built on the GPU)."""
        lib = load()
        t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
        self.num_tris = t.shape[0]
        gid = ctypes.c_uint64(0)
        _check(lib.pgpu_geometry_create_ex(_ptr(t, ctypes.c_float), t.shape[0], float(max_origin_abs),
                                           BUILDERS[builder], ctypes.byref(gid)))
        self.id = gid.value

    def export(self):
        """(nodes uint32 [N, 20], leaf triangles as a structured array) copied from the device."""
        nn, nt = ctypes.c_uint64(), ctypes.c_uint64()
        _check(load().pgpu_geometry_export(self.id, None, None, ctypes.byref(nn), ctypes.byref(nt)))
        nodes = np.empty((nn.value, 20), np.uint32)
        tris = np.empty(nt.value, LEAF_TRI_DTYPE)
        _check(load().pgpu_geometry_export(self.id, nodes.ctypes.data_as(ctypes.c_void_p),
                                           tris.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nn), ctypes.byref(nt)))
        return nodes, tris

    def close(self) -> None:
        if self.id:
            _check(load().pgpu_geometry_destroy(self.id))
            self.id = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def stats(self) -> dict:
        nn, nt = ctypes.c_uint64(), ctypes.c_uint64()
        depth, secs = ctypes.c_int32(), ctypes.c_double()
        _check(load().pgpu_geometry_stats(self.id, ctypes.byref(nn), ctypes.byref(nt),
                                          ctypes.byref(depth), ctypes.byref(secs)))
        return {"num_nodes": nn.value, "num_tris": nt.value, "max_depth": depth.value,
                "build_seconds": secs.value}

    def closest(self, rays: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = r.shape[0]
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        bary = np.empty((n, 3), np.float32)
        _check(load().pgpu_trace_closest(self.id, _ptr(r, ctypes.c_float), n, _ptr(prim, ctypes.c_int32),
                                         _ptr(t, ctypes.c_float), _ptr(bary, ctypes.c_float)))
        return prim, t, bary

    def occluded(self, rays: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.empty(r.shape[0], np.int32)
        _check(load().pgpu_trace_any(self.id, _ptr(r, ctypes.c_float), r.shape[0], _ptr(out, ctypes.c_int32)))
        return out

    def counts(self, rays: np.ndarray, any_hit: bool = False) -> Tuple[float, float]:
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        nodes, tris = ctypes.c_double(), ctypes.c_double()
        _check(load().pgpu_trace_counts(self.id, _ptr(r, ctypes.c_float), r.shape[0], int(any_hit),
                                        ctypes.byref(nodes), ctypes.byref(tris)))
        return nodes.value, tris.value


def bsdf_eval(cases: np.ndarray, normals: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(cases, np.float32).reshape(-1, 19)
    nrm = np.ascontiguousarray(normals, np.float32).reshape(-1, 6)
    out = np.empty((c.shape[0], 16), np.float32)
    _check(load().pgpu_bsdf_eval(_ptr(c, ctypes.c_float), _ptr(nrm, ctypes.c_float), c.shape[0],
                                 _ptr(out, ctypes.c_float)))
    return out


FILM_FILTERS = {"gaussian": 1, "mitchell-netravali": 2, "blackman-harris": 3}


def film_splat(sample_filter: str, width: int, height: int, samples: np.ndarray) -> np.ndarray:
    """(R, G, B, W) sums float64 [height, width, 4] of samples [n, 5] = raster x, raster y, r, g, b
    splatted through one of the 4 x 4 filters on the GPU."""
    smp = np.ascontiguousarray(samples, np.float32).reshape(-1, 5)
    sums = np.empty((height, width, 4), np.float64)
    _check(load().pgpu_film_splat(FILM_FILTERS[sample_filter], width, height, _ptr(smp, ctypes.c_float), smp.shape[0],
                                  _ptr(sums, ctypes.c_double)))
    return sums


def guide_forward(params: np.ndarray, features: np.ndarray) -> np.ndarray:
    """Raw outputs [n, 40] of the guiding network (tensor-core forward pass) for features [n, 7]."""
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    f = np.ascontiguousarray(features, np.float32).reshape(-1, 7)
    out = np.empty((f.shape[0], 40), np.float32)
    _check(load().pgpu_guide_forward(_ptr(p, ctypes.c_float), _ptr(f, ctypes.c_float), f.shape[0],
                                     _ptr(out, ctypes.c_float)))
    return out


def guide_mixture(params: np.ndarray, features: np.ndarray) -> np.ndarray:
    """Decoded mixtures [n, 8, 6] of the guiding network for features [n, 7]: per lobe (weight,
    mean xyz, kappa, weight x vMF normalisation), as the renderer samples them."""
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    f = np.ascontiguousarray(features, np.float32).reshape(-1, 7)
    out = np.empty((f.shape[0], 8, 6), np.float32)
    _check(load().pgpu_guide_mixture(_ptr(p, ctypes.c_float), _ptr(f, ctypes.c_float), f.shape[0],
                                     _ptr(out, ctypes.c_float)))
    return out


def guide_gradients(params, features, dirs, weights, cuda_cores: bool = False):
    """(loss, gradient [29480]) of the guiding loss on one batch (GPU): backward pass on the tensor
    cores, or with cuda_cores in FP32 on the CUDA cores."""
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    f = np.ascontiguousarray(features, np.float32).reshape(-1, 7)
    d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    w = np.ascontiguousarray(weights, np.float32).reshape(-1)
    g = np.empty_like(p)
    loss = ctypes.c_float()
    _check(load().pgpu_guide_gradients_ex(_ptr(p, ctypes.c_float), _ptr(f, ctypes.c_float), _ptr(d, ctypes.c_float),
                                          _ptr(w, ctypes.c_float), f.shape[0], 1 if cuda_cores else 0,
                                          ctypes.byref(loss), _ptr(g, ctypes.c_float)))
    return loss.value, g


def guide_train(params, features, dirs, weights, steps, batch, lr=1e-2):
    """Adam-trains a copy of params on the data set; returns (params, per-step losses)."""
    p = np.array(params, np.float32).reshape(-1)
    f = np.ascontiguousarray(features, np.float32).reshape(-1, 7)
    d = np.ascontiguousarray(dirs, np.float32).reshape(-1, 3)
    w = np.ascontiguousarray(weights, np.float32).reshape(-1)
    losses = np.empty(steps, np.float32)
    _check(load().pgpu_guide_train(_ptr(p, ctypes.c_float), _ptr(f, ctypes.c_float), _ptr(d, ctypes.c_float),
                                   _ptr(w, ctypes.c_float), f.shape[0], steps, batch, lr, _ptr(losses, ctypes.c_float)))
    return p, losses


MATTE, CONDUCTOR, DIELECTRIC = 0, 1, 2
BNEEPT, BVPT, BVPTDL = 0, 1, 2
# sample-filter names of the reference's SDL (sdl_sample_filter_type.h) -> pgpu_scene_set_filter
FILTERS = {"box": 0, "gaussian": 1, "mn": 2, "bh": 3}
# phGpuSetDomePdf / pgpu_scene_set_dome_pdf modes
DOME_PDF = {"reference": 0, "exact": 1}


def flatten_scene(scene):
    """Flat arrays of a ``scenes.Scene`` in the layout pgpu_scene_create expects."""
    tris, tri_mat, tri_em, mats, ems = [], [], [], [], []
    for g in scene.groups:
        m = g.material
        kind = {"matte": MATTE, "conductor": CONDUCTOR, "dielectric": DIELECTRIC}[m.kind]
        c = m.albedo if m.kind == "matte" else m.f0
        mats.append([kind, c[0], c[1], c[2], m.roughness, m.ior_outer, m.ior_inner, 0.0])
        n = g.tris.shape[0]
        tris.append(np.asarray(g.tris, np.float32).reshape(n, 9))
        tri_mat.append(np.full(n, len(mats) - 1, np.uint32))
        if g.radiance is not None:
            ems.append([g.radiance[0], g.radiance[1], g.radiance[2], 0.0])
            tri_em.append(np.full(n, len(ems), np.uint32))
        else:
            tri_em.append(np.zeros(n, np.uint32))
    if scene.env_image is not None:
        raise ValueError("the flat scene ABI takes constant environments only; render image domes through the "
                         "Photon C API (SDL image-dome)")
    if scene.env_radiance is not None:
        ems.append([scene.env_radiance[0], scene.env_radiance[1], scene.env_radiance[2], 1.0])
    cam = np.array(list(scene.cam_pos) + list(scene.cam_dir) + list(scene.cam_up)
                   + [scene.fov_deg, scene.width, scene.height], np.float32)
    return (np.ascontiguousarray(np.concatenate(tris)), np.concatenate(tri_mat), np.concatenate(tri_em),
            np.asarray(mats, np.float32).reshape(-1, 8), np.asarray(ems, np.float32).reshape(-1, 4), cam)


def render_scenes(render_scenes, spp, max_bounces=10000, estimator=BNEEPT, seed=42, concurrency=4) -> float:
    """pgpu_scenes_render: renders RenderScenes together (spp[i] more samples each), up to
    `concurrency` at a time on their own streams; returns the batch's device span in ms."""
    ids = np.array([rs.id for rs in render_scenes], np.uint64)
    counts = np.array(spp, np.uint32)
    ms = ctypes.c_float()
    _check(load().pgpu_scenes_render(_ptr(ids, ctypes.c_uint64), len(ids), _ptr(counts, ctypes.c_uint32), max_bounces,
                                     estimator, seed, concurrency, ctypes.byref(ms)))
    return ms.value


def render_scenes_wavefront(render_scenes, spp, max_bounces=10000, estimator=BNEEPT, seed=42) -> float:
    """pgpu_scenes_render_wavefront: renders RenderScenes (spp[i] more samples each) as one
    wavefront -- one path pool and one launch per kernel per iteration for all of them; returns
    the batch's device ms."""
    ids = np.array([rs.id for rs in render_scenes], np.uint64)
    counts = np.array(spp, np.uint32)
    ms = ctypes.c_float()
    _check(load().pgpu_scenes_render_wavefront(_ptr(ids, ctypes.c_uint64), len(ids), _ptr(counts, ctypes.c_uint32),
                                               max_bounces, estimator, seed, ctypes.byref(ms)))
    return ms.value


def autotune_wavefront(render_scenes, spp, max_bounces=10000, estimator=BNEEPT) -> dict:
    """pgpu_scenes_autotune_wavefront: launch shapes of the one-wavefront render of these scenes."""
    ids = np.array([rs.id for rs in render_scenes], np.uint64)
    counts = np.array(spp, np.uint32)
    cfg = np.zeros(4, np.uint32)
    ms = np.zeros(4, np.float32)
    _check(load().pgpu_scenes_autotune_wavefront(_ptr(ids, ctypes.c_uint64), len(ids), _ptr(counts, ctypes.c_uint32),
                                                 max_bounces, estimator, _ptr(cfg, ctypes.c_uint32),
                                                 _ptr(ms, ctypes.c_float)))
    return {"capacity": int(cfg[0]), "refill": int(cfg[1]), "blocks_per_sm": int(cfg[2]), "leaf_tris": int(cfg[3]),
            "ms_default": float(ms[0]), "ms_tuned": float(ms[1]), "trials": int(ms[2])}


class RenderScene:
    """A scene resident on the GPU with its FP64 film (pgpu_scene_*)."""

    def __init__(self, scene, builder: str = "sah"):
        lib = load()
        tris, tri_mat, tri_em, mats, ems, cam = flatten_scene(scene)
        self.width, self.height = scene.width, scene.height
        sid = ctypes.c_uint64(0)
        em_ptr = _ptr(ems, ctypes.c_float) if ems.size else None
        _check(lib.pgpu_scene_create_ex(_ptr(tris, ctypes.c_float), _ptr(tri_mat, ctypes.c_uint32),
                                        _ptr(tri_em, ctypes.c_uint32), tris.shape[0],
                                        _ptr(mats, ctypes.c_float), mats.shape[0], em_ptr, ems.shape[0],
                                        _ptr(cam, ctypes.c_float), BUILDERS[builder], ctypes.byref(sid)))
        self.id = sid.value

    def close(self):
        if self.id:
            _check(load().pgpu_scene_destroy(self.id))
            self.id = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def render(self, spp, max_bounces=10000, estimator=BNEEPT, seed=42, first_sample=0):
        ms = ctypes.c_float()
        rays, shadow = ctypes.c_uint64(), ctypes.c_uint64()
        _check(load().pgpu_scene_render(self.id, spp, max_bounces, estimator, seed, first_sample,
                                        ctypes.byref(ms), ctypes.byref(rays), ctypes.byref(shadow)))
        return {"ms": ms.value, "rays": rays.value, "shadow_rays": shadow.value}

    def film(self, with_sums: bool = True):
        """(developed float32 [H, W, 3], FP64 sums [H, W, 4] = R, G, B, W or None, spp)."""
        rgb = np.empty((self.height, self.width, 3), np.float32)
        sums = np.empty((self.height, self.width, 4), np.float64) if with_sums else None
        spp = ctypes.c_uint64()
        _check(load().pgpu_scene_film(self.id, _ptr(rgb, ctypes.c_float),
                                      _ptr(sums, ctypes.c_double) if with_sums else None, ctypes.byref(spp)))
        return rgb, sums, spp.value

    def clear(self):
        _check(load().pgpu_scene_clear(self.id))

    def set_dome_pdf(self, mode: str) -> None:
        """Environment sample densities: "reference" (default) or "exact"."""
        _check(load().pgpu_scene_set_dome_pdf(self.id, DOME_PDF[mode]))

    def set_filter(self, name: str) -> None:
        """Sample filter of the film ("box", "gaussian", "mn", "bh"); clears the film."""
        _check(load().pgpu_scene_set_filter(self.id, FILTERS[name]))

    def profile(self, spp, max_bounces=10000, estimator=BNEEPT, seed=42):
        """Per-kernel device ms of a timed render into a scratch film."""
        ms = np.zeros(7, np.float64)
        _check(load().pgpu_scene_profile(self.id, spp, max_bounces, estimator, seed, _ptr(ms, ctypes.c_double)))
        keys = ["prepare_ms", "regen_ms", "extend_ms", "shade_ms", "shadow_ms", "guide_infer_ms", "guide_train_ms"]
        return dict(zip(keys, ms.tolist()))

    def autotune(self, spp, max_bounces=10000, estimator=BNEEPT, rebuild=True, cache_path=None,
                 ignore_cache=False) -> dict:
        """pgpu_scene_autotune: picks the scene's launch shapes; returns them with the calibration
        render's device ms under the defaults and under the choice."""
        cfg = np.zeros(4, np.uint32)
        ms = np.zeros(4, np.float32)
        flags = (1 if rebuild else 0) | (2 if ignore_cache else 0)
        _check(load().pgpu_scene_autotune(self.id, spp, max_bounces, estimator, flags,
                                          cache_path.encode() if cache_path else None, _ptr(cfg, ctypes.c_uint32),
                                          _ptr(ms, ctypes.c_float)))
        return {"capacity": int(cfg[0]), "refill": int(cfg[1]), "blocks_per_sm": int(cfg[2]), "leaf_tris": int(cfg[3]),
                "ms_default": float(ms[0]), "ms_tuned": float(ms[1]), "trials": int(ms[2]), "from_cache": bool(ms[3])}

    def set_launch(self, capacity=1 << 21, refill=8, blocks_per_sm=8, leaf_tris=3) -> None:
        cfg = np.array([capacity, refill, blocks_per_sm, leaf_tris], np.uint32)
        _check(load().pgpu_scene_set_launch(self.id, _ptr(cfg, ctypes.c_uint32)))

    def launch(self) -> dict:
        cfg = np.zeros(4, np.uint32)
        _check(load().pgpu_scene_get_launch(self.id, _ptr(cfg, ctypes.c_uint32)))
        return {"capacity": int(cfg[0]), "refill": int(cfg[1]), "blocks_per_sm": int(cfg[2]), "leaf_tris": int(cfg[3])}

    def light_pmf(self):
        """(pmf float32 [E], alias-table pmf float64 [E]) of the scene's emitters (pgpu_scene_light_pmf)."""
        lib = load()
        n = ctypes.c_uint32(0)
        _check(lib.pgpu_scene_light_pmf(self.id, None, None, ctypes.byref(n)))
        pmf = np.zeros(n.value, np.float32)
        alias = np.zeros(n.value, np.float64)
        if n.value:
            _check(lib.pgpu_scene_light_pmf(self.id, _ptr(pmf, ctypes.c_float), _ptr(alias, ctypes.c_double),
                                            ctypes.byref(n)))
        return pmf, alias

    def light_pdf(self, targets: np.ndarray, points: np.ndarray, prims: np.ndarray) -> np.ndarray:
        """NEE solid-angle densities for receiving points, light points and light-triangle indices
        (pgpu_scene_light_pdf)."""
        q = np.ascontiguousarray(np.concatenate([np.asarray(targets, np.float32).reshape(-1, 3),
                                                 np.asarray(points, np.float32).reshape(-1, 3)], axis=1))
        pr = np.ascontiguousarray(prims, np.uint32)
        out = np.zeros(q.shape[0], np.float32)
        _check(load().pgpu_scene_light_pdf(self.id, _ptr(q, ctypes.c_float), _ptr(pr, ctypes.c_uint32), q.shape[0],
                                           _ptr(out, ctypes.c_float)))
        return out

    def launches(self) -> int:
        """Kernels launched by the last render (pgpu_scene_launches)."""
        n = ctypes.c_uint64()
        _check(load().pgpu_scene_launches(self.id, ctypes.byref(n)))
        return n.value

    def count(self, spp, max_bounces=10000, estimator=BNEEPT, seed=42):
        """Traversal work of a render into a scratch film (pgpu_scene_count)."""
        c = np.zeros(7, np.uint64)
        _check(load().pgpu_scene_count(self.id, spp, max_bounces, estimator, seed, _ptr(c, ctypes.c_uint64)))
        keys = ["rays", "shadow_rays", "nodes_closest", "tris_closest", "nodes_any", "tris_any", "iterations"]
        return dict(zip(keys, (int(x) for x in c)))

    def set_guiding(self, enabled=True, train=True, alpha=0.5, lr=1e-2, batch=16384):
        _check(load().pgpu_scene_set_guiding(self.id, int(enabled), int(train), alpha, lr, batch))

    def set_guiding_depth(self, depth: int) -> None:
        """Guide the first `depth` vertices of every path (default 1; 0 = every vertex)."""
        _check(load().pgpu_scene_set_guiding_depth(self.id, depth))

    def guide_reset(self):
        _check(load().pgpu_scene_guide_reset(self.id))

    def guide_info(self, with_params=False):
        loss = ctypes.c_float()
        guided = ctypes.c_uint64()
        ms = np.zeros(7, np.float64)
        params = np.empty(29480, np.float32) if with_params else None
        _check(load().pgpu_scene_guide_info(self.id, ctypes.byref(loss), ctypes.byref(guided), _ptr(ms, ctypes.c_double),
                                            _ptr(params, ctypes.c_float) if with_params else None))
        keys = ["prepare_ms", "regen_ms", "extend_ms", "shade_ms", "shadow_ms", "guide_infer_ms", "guide_train_ms"]
        out = {"loss": loss.value, "guided_vertices": guided.value, "kernel_ms": dict(zip(keys, ms.tolist()))}
        if with_params:
            out["params"] = params
        return out


# ----------------------------------------------------------------------------------------------
# Photon C API (ph_c_core.h) declared on the same library.

_u8pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_ubyte))
_f32pp = ctypes.POINTER(_f32p)
_charpp = ctypes.POINTER(ctypes.c_char_p)

PH_SIGNATURES = [
    ("phConfigRendererResourceDirectory", None, [ctypes.c_char_p]),
    ("phInit", ctypes.c_int, []),
    ("phExit", ctypes.c_int, []),
    ("phCreateEngine", None, [_u64p, ctypes.c_uint32]),
    ("phSetNumRenderThreads", None, [ctypes.c_uint64, ctypes.c_uint32]),
    ("phEnterCommand", None, [ctypes.c_uint64, ctypes.c_char_p]),
    ("phLoadCommands", ctypes.c_int, [ctypes.c_uint64, ctypes.c_char_p]),
    ("phRender", None, [ctypes.c_uint64]),
    ("phUpdate", None, [ctypes.c_uint64]),
    ("phGetRenderDimension", None, [ctypes.c_uint64, _u32p, _u32p]),
    ("phGetObservableRenderData", None, [ctypes.c_uint64, ctypes.c_void_p]),
    ("phDeleteEngine", None, [ctypes.c_uint64]),
    ("phSetWorkingDirectory", None, [ctypes.c_uint64, ctypes.c_char_p]),
    ("phAquireFrame", None, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    ("phAquireFrameRaw", None, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    ("phCreateFrame", None, [_u64p, ctypes.c_uint32, ctypes.c_uint32]),
    ("phGetFrameDimension", None, [ctypes.c_uint64, _u32p, _u32p]),
    ("phGetFrameRgbData", None, [ctypes.c_uint64, _f32pp]),
    ("phDeleteFrame", None, [ctypes.c_uint64]),
    ("phLoadFrame", ctypes.c_int, [ctypes.c_uint64, ctypes.c_char_p]),
    ("phSaveFrame", ctypes.c_int, [ctypes.c_uint64, ctypes.c_char_p, ctypes.c_void_p]),
    ("phSaveFrameToBuffer", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p]),
    ("phFrameOpAbsDifference", None, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    ("phFrameOpMSE", ctypes.c_float, [ctypes.c_uint64, ctypes.c_uint64]),
    ("phCreateBuffer", None, [_u64p]),
    ("phGetBufferBytes", None, [ctypes.c_uint64, _u8pp, ctypes.POINTER(ctypes.c_size_t)]),
    ("phDeleteBuffer", None, [ctypes.c_uint64]),
    ("phAsyncGetRenderProgress", None, [ctypes.c_uint64, ctypes.c_void_p]),
    ("phAsyncGetRenderStatistics", None, [ctypes.c_uint64, _f32p, _f32p]),
    ("phAsyncGetRenderState", None, [ctypes.c_uint64, ctypes.c_void_p]),
    ("phAsyncPollUpdatedFrameRegion", ctypes.c_int, [ctypes.c_uint64, ctypes.c_void_p]),
    ("phAsyncPollUpdatedFrameRegions", ctypes.c_size_t,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t]),
    ("phAsyncPollMergedUpdatedFrameRegions", ctypes.c_size_t,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]),
    ("phAsyncPeekFrame", None,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.c_uint64]),
    ("phAsyncPeekFrameRaw", None,
     [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
      ctypes.c_uint64]),
    ("phGpuGetErrors", ctypes.c_int, [ctypes.c_uint64, _charpp]),
    ("phGpuSetMaxRayBounces", None, [ctypes.c_uint64, ctypes.c_uint32]),
    ("phGpuSetSeed", None, [ctypes.c_uint64, ctypes.c_uint64]),
    ("phGpuSetGuiding", None, [ctypes.c_uint64, ctypes.c_int]),
    ("phGpuSetBvhBuilder", None, [ctypes.c_uint64, ctypes.c_uint32]),
    ("phGpuSetDomePdf", None, [ctypes.c_uint64, ctypes.c_uint32]),
    ("phGpuSetSurfaceRefine", None, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32]),
    ("phGpuClearFilm", None, [ctypes.c_uint64]),
    ("phGpuGetRenderInfo", None, [ctypes.c_uint64, _dblp, _u64p, _u64p, _u64p, _dblp]),
    ("phGpuGetLaunchCount", ctypes.c_uint64, [ctypes.c_uint64]),
    ("phGpuProfileRender", None, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, _dblp]),
    ("phGpuAutotune", ctypes.c_int, [ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint32, _u32p, _f32p]),
]


class CookedScene:
    """Result of pgpu_sdl_cook: what phUpdate would upload, computed on the host."""

    def __init__(self, sdl_text: str, working_dir: str = "."):
        lib = load()
        txt = sdl_text.encode()
        wd = working_dir.encode()
        n = ctypes.c_uint64()
        nm, ne = ctypes.c_uint32(), ctypes.c_uint32()
        dims = np.zeros(5, np.uint32)
        _check(lib.pgpu_sdl_cook(txt, wd, ctypes.byref(n), ctypes.byref(nm), ctypes.byref(ne),
                                 _ptr(dims, ctypes.c_uint32), None, None, None, None, None))
        self.tris = np.empty((n.value, 3, 3), np.float32)
        self.tri_material = np.empty(n.value, np.uint32)
        self.tri_emitter = np.empty(n.value, np.uint32)
        self.emitters = np.empty((ne.value, 4), np.float32)
        self.camera = np.empty(16, np.float32)
        _check(lib.pgpu_sdl_cook(txt, wd, ctypes.byref(n), ctypes.byref(nm), ctypes.byref(ne),
                                 _ptr(dims, ctypes.c_uint32), _ptr(self.tris, ctypes.c_float),
                                 _ptr(self.tri_material, ctypes.c_uint32), _ptr(self.tri_emitter, ctypes.c_uint32),
                                 _ptr(self.emitters, ctypes.c_float) if ne.value else None,
                                 _ptr(self.camera, ctypes.c_float)))
        self.num_materials = nm.value
        self.width, self.height, self.spp, self.estimator, self.sample_filter = (int(x) for x in dims)


class FrameRegion(ctypes.Structure):
    """PhFrameRegionInfo (ph_c_core_types.h)."""

    _fields_ = [("x", ctypes.c_uint32), ("y", ctypes.c_uint32), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("status", ctypes.c_int)]


REGION_FINISHED = 1
REGION_UPDATING = 2


class PhotonEngine:
    """The Photon C API (phCreateEngine ... phAquireFrameRaw) on this library."""

    def __init__(self, threads: int = 1):
        lib = load()
        if not lib.phInit():
            raise PhotonGpuError(PG_ERR_NO_DEVICE, "phInit failed (no CUDA device?)")
        eid = ctypes.c_uint64()
        lib.phCreateEngine(ctypes.byref(eid), threads)
        self.id = eid.value

    def enter(self, text: str) -> None:
        load().phEnterCommand(self.id, text.encode())

    def load_file(self, path: str) -> bool:
        return bool(load().phLoadCommands(self.id, path.encode()))

    def set_working_directory(self, path: str) -> None:
        load().phSetWorkingDirectory(self.id, path.encode())

    def set_max_bounces(self, n: int) -> None:
        load().phGpuSetMaxRayBounces(self.id, n)

    def set_guiding(self, enabled: bool) -> None:
        load().phGpuSetGuiding(self.id, 1 if enabled else 0)

    def set_bvh_builder(self, builder: str = "sah") -> None:
        load().phGpuSetBvhBuilder(self.id, BUILDERS[builder])

    def set_dome_pdf(self, mode: str = "reference") -> None:
        """phGpuSetDomePdf: environment sample densities as the reference computes them, or exact."""
        load().phGpuSetDomePdf(self.id, DOME_PDF[mode])

    def set_surface_refine(self, mode: str = "iterative", delta: float = 2e-4, iterations: int = 1) -> None:
        """phGpuSetSurfaceRefine: the reference's RefineMode (manual / empirical / iterative)."""
        m = {"manual": 0, "empirical": 1, "iterative": 2}[mode]
        load().phGpuSetSurfaceRefine(self.id, m, delta, iterations)

    def set_seed(self, seed: int) -> None:
        load().phGpuSetSeed(self.id, seed)

    def update(self) -> None:
        load().phUpdate(self.id)
        self._raise_errors()

    def render(self) -> None:
        load().phRender(self.id)
        self._raise_errors()

    def clear_film(self) -> None:
        load().phGpuClearFilm(self.id)

    def errors(self) -> str:
        msg = ctypes.c_char_p()
        load().phGpuGetErrors(self.id, ctypes.byref(msg))
        return (msg.value or b"").decode(errors="replace")

    def _raise_errors(self) -> None:
        err = self.errors()
        fatal = [line for line in err.splitlines() if "failed" in line]
        if fatal:
            raise PhotonGpuError(PG_ERR_SCENE, "\n".join(fatal))

    def dimension(self):
        w, h = ctypes.c_uint32(), ctypes.c_uint32()
        load().phGetRenderDimension(self.id, ctypes.byref(w), ctypes.byref(h))
        return w.value, h.value

    def info(self) -> dict:
        ms, upd = ctypes.c_double(), ctypes.c_double()
        paths, rays, shadow = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        load().phGpuGetRenderInfo(self.id, ctypes.byref(ms), ctypes.byref(paths), ctypes.byref(rays),
                                  ctypes.byref(shadow), ctypes.byref(upd))
        return {"device_ms": ms.value, "paths": paths.value, "rays": rays.value,
                "shadow_rays": shadow.value, "update_seconds": upd.value}

    def launch_count(self) -> int:
        return int(load().phGpuGetLaunchCount(self.id))

    def autotune(self, cache_path=None, rebuild=True, ignore_cache=False) -> dict:
        """phGpuAutotune: launch shapes of the updated scene for the session's spp and estimator."""
        cfg = np.zeros(4, np.uint32)
        ms = np.zeros(4, np.float32)
        flags = (1 if rebuild else 0) | (2 if ignore_cache else 0)
        ok = load().phGpuAutotune(self.id, cache_path.encode() if cache_path else None, flags,
                                  _ptr(cfg, ctypes.c_uint32), _ptr(ms, ctypes.c_float))
        if not ok:
            raise PhotonGpuError(PG_ERR_SCENE, self.errors())
        return {"capacity": int(cfg[0]), "refill": int(cfg[1]), "blocks_per_sm": int(cfg[2]), "leaf_tris": int(cfg[3]),
                "ms_default": float(ms[0]), "ms_tuned": float(ms[1]), "trials": int(ms[2]), "from_cache": bool(ms[3])}

    def profile(self, mode: int, spp: int) -> dict:
        """phGpuProfileRender: mode 1 per-kernel timing, mode 2 traversal counting."""
        stats = np.zeros(14, np.float64)
        load().phGpuProfileRender(self.id, mode, spp, _ptr(stats, ctypes.c_double))
        self._raise_errors()
        keys = ["prepare_ms", "regen_ms", "extend_ms", "shade_ms", "shadow_ms", "total_ms", "paths",
                "rays", "shadow_rays", "iterations", "nodes_closest", "tris_closest", "nodes_any", "tris_any"]
        return dict(zip(keys, stats.tolist()))

    def frame(self) -> np.ndarray:
        """phCreateFrame + phAquireFrameRaw + phGetFrameRgbData: float32 [H, W, 3], row 0 bottom."""
        lib = load()
        w, h = self.dimension()
        fid = ctypes.c_uint64()
        lib.phCreateFrame(ctypes.byref(fid), w, h)
        try:
            lib.phAquireFrameRaw(self.id, 0, fid.value)
            data = _f32p()
            lib.phGetFrameRgbData(fid.value, ctypes.byref(data))
            return np.ctypeslib.as_array(data, shape=(h, w, 3)).copy()
        finally:
            lib.phDeleteFrame(fid.value)

    def poll_region(self) -> Optional[Tuple[int, int, int, int, int]]:
        """phAsyncPollUpdatedFrameRegion: (x, y, width, height, status) or None."""
        r = FrameRegion()
        if load().phAsyncPollUpdatedFrameRegion(self.id, ctypes.byref(r)):
            return (r.x, r.y, r.width, r.height, r.status)
        return None

    def poll_regions(self, max_regions: int = 64, merged: bool = False):
        """phAsyncPollUpdatedFrameRegions (or the merged variant): a list of (x, y, w, h, status)."""
        arr = (FrameRegion * max_regions)()
        lib = load()
        if merged:
            n = lib.phAsyncPollMergedUpdatedFrameRegions(self.id, 0, 1, arr, max_regions)
        else:
            n = lib.phAsyncPollUpdatedFrameRegions(self.id, 0, arr, max_regions)
        return [(r.x, r.y, r.width, r.height, r.status) for r in arr[:n]]

    def progress(self) -> Tuple[int, int, int]:
        """phAsyncGetRenderProgress: (total work, work done, elapsed ms) in samples per pixel."""
        class _Progress(ctypes.Structure):
            _fields_ = [("total", ctypes.c_uint64), ("done", ctypes.c_uint64), ("ms", ctypes.c_uint64)]
        p = _Progress()
        load().phAsyncGetRenderProgress(self.id, ctypes.byref(p))
        return p.total, p.done, p.ms

    def peek(self, x: int = 0, y: int = 0, width: int = 0, height: int = 0) -> np.ndarray:
        """phAsyncPeekFrameRaw of a rectangle (the whole frame by default) into a new frame:
        float32 [H, W, 3] of the full frame, pixels outside the rectangle 0."""
        lib = load()
        w, h = self.dimension()
        fid = ctypes.c_uint64()
        lib.phCreateFrame(ctypes.byref(fid), w, h)
        try:
            lib.phAsyncPeekFrameRaw(self.id, 0, x, y, width or w, height or h, fid.value)
            data = _f32p()
            lib.phGetFrameRgbData(fid.value, ctypes.byref(data))
            return np.ctypeslib.as_array(data, shape=(h, w, 3)).copy()
        finally:
            lib.phDeleteFrame(fid.value)

    def close(self) -> None:
        if self.id:
            load().phDeleteEngine(self.id)
            self.id = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


PG_ERR_SCENE = 6
PG_ERR_NO_DEVICE = 7


def _declare_ph_api(lib: ctypes.CDLL) -> None:
    for name, res, args in PH_SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
