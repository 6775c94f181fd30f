"""Reference renders for the image-parity tests, made by the reference CPU renderer itself.

Run in the build container after building the oracle (``make -f oracle/Makefile.ref REF=<reference sources> -j8``):

    python tests/golden/make_golden_images.py [workload ...]

With workload names given, only those are re-rendered and the rest of images.npz is kept.

For each workload below the scene is generated by photon-v2_b200/scenes.py, written as SDL, and
rendered with oracle/_ref/ph_ref_render (phLoadCommands -> phUpdate -> phRender ->
phAquireFrameRaw). The developed frames go to images.npz (float32 [H, W, 3], row 0 = bottom)
together with the spp and bounce cap used. Every workload is small (32 x 32 to 128 x 128) and rendered
with many samples so that its own noise stays well below the parity bar.
"""

import os
import subprocess
import sys
import tempfile

import dataclasses

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "photon-v2_b200"))

import scenes  # noqa: E402

RENDER_TOOL = os.path.join(ROOT, "oracle", "_ref", "ph_ref_render")

# name -> (scene factory, spp, max bounces[, the reference's RefineMode in its EngineConfig.ini])
WORKLOADS = {
    "cornell_bneept": (lambda spp: scenes.cornell(64, 64, spp, 8, "bneept"), 8192, 8),
    "cornell_bvpt": (lambda spp: scenes.cornell(64, 64, spp, 8, "bvpt"), 8192, 8),
    "cornell_bvptdl": (lambda spp: scenes.cornell(64, 64, spp, 8, "bvptdl"), 8192, 8),
    # the grey furnace (32 x 32): the reference's finite-dome densities bias it above 0.5
    "furnace_bneept_ref": (lambda spp: scenes.furnace(spp), 8192, 10000),
    # a lat-long image dome (sky with a small sun), rotated 60 degrees about +y
    "ggx_sphere_envmap_bneept": (lambda spp: dataclasses.replace(
        scenes.ggx_sphere(level=3, width=64, height=64, spp=spp, max_bounces=10),
        env_radiance=None, env_image=scenes.sky_image(), env_rotation=((0.0, 1.0, 0.0), 60.0)), 8192, 10),
    # the reference's other sample filters (sample-filter of the path-tracing visualizer)
    "cornell_bneept_gaussian": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                                sample_filter="gaussian"), 8192, 8),
    "cornell_bneept_mn": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                          sample_filter="mn"), 8192, 8),
    "cornell_bneept_bh": (lambda spp: dataclasses.replace(scenes.cornell(64, 64, spp, 8, "bneept"),
                                                          sample_filter="bh"), 8192, 8),
    "cornell_glossy_bneept": (lambda spp: scenes.cornell_glossy(64, 64, spp, 8, "bneept"), 8192, 8),
    "ggx_sphere_env_bneept": (lambda spp: scenes.ggx_sphere(level=3, width=64, height=64, spp=spp,
                                                            max_bounces=10), 4096, 10),
    "cornell_glossy_bneept_empirical": (lambda spp: scenes.cornell_glossy(64, 64, spp, 8, "bneept"), 8192, 8,
                                        "empirical"),
    "ggx_sphere_bneept_manual": (lambda spp: scenes.ggx_sphere(level=3, width=64, height=64, spp=spp,
                                                               max_bounces=10), 4096, 10, "manual"),
    # the benchmarked configurations' geometry at reduced resolution:
    # the 1M-triangle GGX scene (1,310,726 triangles, 2 quad lights + environment, depth 10) at
    # 64 x 64 and 65,536 spp -- the converged reference its parity and error are stated against
    "c2_ggx1m_bneept": (lambda spp: scenes.ggx_sphere(level=8, width=64, height=64, spp=spp,
                                                      max_bounces=10), 65536, 10),
    # the slit-light room, full 2M triangles with its dielectric boxes, 32 x 32
    "slit_room_bneept": (lambda spp: scenes.slit_room(32, 32, spp, 10), 262144, 10),
    # the same room with every box Lambertian, and with glass at depth 2: light through the slit
    # without the caustics of the glass boxes, whose rare, very bright paths make the full room's
    # image mean converge slowly
    "slit_room_matte_bneept": (lambda spp: scenes.slit_room(32, 32, spp, 10, glass_fraction=0.0), 16384, 10),
    "slit_room_depth2_bneept": (lambda spp: scenes.slit_room(32, 32, spp, 2), 262144, 2),
    # a 40 x 40-block tile of the many-light city (174,802 triangles) with 1,000 lights, depth 12
    "city_tile_bneept": (lambda spp: scenes.city(64, 64, spp, 12, blocks=40, num_lights=1000), 16384, 12),
}


def render(scene: scenes.Scene, max_bounces: int, threads: int, refine_mode: str = "iterative") -> np.ndarray:
    with tempfile.TemporaryDirectory() as tmp:
        # the reference reads its surface refiner's mode from ./Config/EngineConfig.ini at phInit
        os.makedirs(os.path.join(tmp, "Config"), exist_ok=True)
        with open(os.path.join(tmp, "Config", "EngineConfig.ini"), "w") as f:
            f.write(f"RefineMode={refine_mode}\nSelfIntersectDelta=2e-04\nNumIterativeSurfaceRefinements=1\n")
        p2 = os.path.join(tmp, "scene.p2")
        with open(p2, "w") as f:
            f.write(scenes.to_sdl(scene))
        scenes.write_env(scene, tmp)
        out = os.path.join(tmp, "out.rgbf32")
        subprocess.run([RENDER_TOOL, p2, str(threads), str(max_bounces), out], check=True, cwd=tmp,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return np.fromfile(out, np.float32).reshape(scene.height, scene.width, 3)


def main() -> None:
    if not os.path.exists(RENDER_TOOL):
        raise SystemExit(f"{RENDER_TOOL} missing: run `make -f oracle/Makefile.ref REF=<reference sources> -j8` first")
    threads = os.cpu_count() or 1
    path = os.path.join(HERE, "images.npz")
    only = sys.argv[1:]
    arrays = dict(np.load(path)) if only and os.path.exists(path) else {}
    for name, (factory, spp, bounces, *mode) in WORKLOADS.items():
        if only and name not in only:
            continue
        img = render(factory(spp), bounces, threads, *mode)
        arrays[name] = img
        arrays[name + "__spp"] = np.array(spp)
        arrays[name + "__bounces"] = np.array(bounces)
        print(f"{name}: mean {img.mean(axis=(0, 1))}")
    np.savez_compressed(path, **arrays)


if __name__ == "__main__":
    main()
