"""Progressive frame regions and previews while phRender runs.

The reference's renderer queues an updated region whenever a worker merges its film into the
main film (UPDATING) and when a work unit completes (FINISHED), and phAsyncPeekFrame develops the
main film as it stands (EqualSamplingRenderer.cpp:119-238, ph_c_core.cpp:517-590); PhotonCLI and
the editor poll these from another thread while phRender blocks. The GPU renderer reports the
whole frame UPDATING at each of its progress points (the host's checks between batches of graph
launches, where every kernel has finished), with a preview of the film over the samples finished so
far, and FINISHED when the render returns.
"""

import threading
import time

import numpy as np
import pytest

import scenes


def _engine(tmp_path, scene):
    import photon_gpu

    p2 = tmp_path / "scene.p2"
    p2.write_text(scenes.to_sdl(scene, mesh_format="ply"))
    scenes.write_meshes(scene, str(tmp_path))
    scenes.write_env(scene, str(tmp_path))
    eng = photon_gpu.PhotonEngine()
    eng.set_working_directory(str(tmp_path))
    assert eng.load_file(str(p2)), eng.errors()
    eng.set_max_bounces(scene.max_bounces)
    eng.set_seed(3)
    eng.update()
    return eng


@pytest.mark.gpu
@pytest.mark.parametrize("sample_filter", ["box", "bh"])
def test_regions_and_previews_while_rendering(gpu_lib, tmp_path, sample_filter):
    """A poller thread sees UPDATING regions of the whole frame while phRender runs and a FINISHED
    region at the end; every preview it peeks is a finite image whose mean is within 5 % of the
    final frame's (an estimate over fewer samples: box film, several hundred thousand paths at the
    first progress point); after the render, a peek returns the final frame bit for bit."""
    import photon_gpu

    scene = scenes.ggx_sphere(level=5, width=256, height=256, spp=2048, max_bounces=10)
    scene.sample_filter = sample_filter
    eng = _engine(tmp_path, scene)
    assert eng.poll_region() is None, "no region before any render"
    regions, previews = [], []
    stop = threading.Event()

    def poller():
        while not stop.is_set():
            r = eng.poll_region()
            if r is None:
                time.sleep(0.0005)
                continue
            regions.append(r)
            if r[4] == photon_gpu.REGION_UPDATING:
                previews.append(eng.peek())

    t = threading.Thread(target=poller)
    t.start()
    try:
        eng.render()
    finally:
        stop.set()
        t.join()
    regions += eng.poll_regions(256)
    final = eng.frame()
    after = eng.peek()
    eng.close()

    w, h = scene.width, scene.height
    status = [r[4] for r in regions]
    print(f"{sample_filter}: {status.count(photon_gpu.REGION_UPDATING)} updating regions, "
          f"{len(previews)} previews, preview means / final: "
          f"{[round(float(p.mean() / final.mean()), 4) for p in previews]}")
    assert all(r[:4] == (0, 0, w, h) for r in regions)
    assert status[-1] == photon_gpu.REGION_FINISHED and status.count(photon_gpu.REGION_FINISHED) == 1
    assert status.count(photon_gpu.REGION_UPDATING) >= 2
    assert np.array_equal(after.view(np.uint32), final.view(np.uint32))
    if sample_filter == "box":
        # box film: every progress point carries the samples finished so far
        assert len(previews) >= 2
        for p in previews:
            assert np.all(np.isfinite(p)) and np.all(p >= 0)
            assert abs(p.mean() / final.mean() - 1.0) < 0.05
    else:
        # 4 x 4 films gain their samples when a pass completes: previews of a single-pass render
        # hold what the film held before it (here nothing)
        for p in previews:
            assert np.all(np.isfinite(p)) and np.all(p >= 0)


@pytest.mark.gpu
def test_progress_and_merged_regions(gpu_lib, tmp_path):
    """phAsyncGetRenderProgress counts samples per pixel done; the merged poll returns at most one
    region (the frame), FINISHED after the render."""
    import photon_gpu

    scene = scenes.ggx_sphere(level=4, width=128, height=128, spp=1024, max_bounces=10)
    eng = _engine(tmp_path, scene)
    eng.render()
    total, done, _ = eng.progress()
    assert total == 1024 and done == 1024
    merged = eng.poll_regions(16, merged=True)
    assert len(merged) == 1 and merged[0][4] == photon_gpu.REGION_FINISHED
    assert eng.poll_regions(16) == []
    eng.close()
