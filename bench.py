"""Throughput benchmark of the GPU BNEEPT path tracer (and of the reference CPU renderer).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads: ggx_1m (default), cornell (256^2, 64 spp, 36 triangles) through the Photon C API;
city, batched and slit_room through the flat scene ABI (see FLAT_WORKLOADS).

Default workload: the 1M-triangle GGX scene -- an icosphere subdivided 8 times (1,310,720
triangles) with seeded 3-octave value-noise radial displacement (5 % of the radius) on a
2-triangle ground, GGX conductors in 64 groups (roughness U[0.05, 0.5], F0 U[0.5, 1]), 2 quad
lights + constant environment 0.1, 1024 x 1024, 256 spp, 10 bounces, FP32 shading with FP64 film.
A step is one full render of that image through the Photon C API (phRender). The scene is
generated in code from fixed seeds (synthetic data, no files).

One JSON line is printed by rank 0. `value` is Mpaths/s (paths = W x H x spp rendered to
completion) over all ranks, timed with CUDA events on the library's stream (max over ranks);
`e2e` is the same metric through phRender + phAquireFrameRaw + phGetFrameRgbData with the
frame copied to host memory, timed on the host clock. Multi-GPU runs are weak-scaled replicas:
every rank renders the full image with its own sample numbering (paths are independent, no
data-path collective).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "photon-v2_b200")
sys.path.insert(0, PKG)

import scenes  # noqa: E402

METRIC = "Mpaths/s and equal-time relMSE: guided vs plain GPU BNEEPT on 1 B200"
REF_RENDER = os.path.join(ROOT, "oracle", "_ref", "ph_ref_render")
PORT_RENDER = os.path.join(ROOT, "oracle", "_build", "ph_port_render")


def workload(name: str) -> scenes.Scene:
    if name == "ggx_1m":
        return scenes.ggx_sphere(level=8, width=1024, height=1024, spp=256, max_bounces=10)
    if name == "cornell":
        return scenes.cornell(256, 256, 64, 8)
    raise SystemExit(f"unknown workload {name}")


def write_scene(scene: scenes.Scene, directory: str) -> str:
    path = os.path.join(directory, "scene.p2")
    with open(path, "w") as f:
        f.write(scenes.to_sdl(scene))
    scenes.write_env(scene, directory)
    return path


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# Reference CPU cost per path on this workload family, measured on the build container's cores
# (1.0 Mpaths/s with 8 threads on the 1M-triangle GGX scene); only used to size the bounded CPU
# sample so that it runs for about `target_seconds` -- the reported number is always measured.
EST_CPU_PATHS_PER_CORE_S = 0.13e6


def cpu_sample(scene: scenes.Scene, tmp: str, target_seconds: float = 12.0, repeats: int = 1,
               force_port: bool = False, paths_per_core_s: float = EST_CPU_PATHS_PER_CORE_S) -> list:
    """Times the reference CPU renderer (or, without it, the oracle port) on a bounded sample of
    the same workload -- the same scene with fewer samples per pixel -- on all host threads.
    Returns one record per repeat (phUpdate untimed, phRender timed)."""
    threads = os.cpu_count() or 1
    tool, kind = (REF_RENDER, "reference") if os.path.exists(REF_RENDER) and not force_port else (PORT_RENDER, "port")
    if not os.path.exists(tool):
        return [{"value": None, "unit": "Mpaths/s", "cores": threads, "kind": kind,
                 "sample": "unavailable: neither oracle/_ref/ph_ref_render nor the port is built"}]
    per_spp_paths = scene.width * scene.height
    spp = int(max(1, min(scene.spp, round(target_seconds * paths_per_core_s * threads / per_spp_paths))))
    s = scenes.Scene(**{**scene.__dict__, "spp": spp})
    d = tempfile.mkdtemp(dir=tmp)
    if kind == "reference":
        scene_file = write_scene(s, d)   # SDL, loaded through phLoadCommands
    else:
        import photon_gpu
        from oracle.port import port as oracle_port

        scene_file = os.path.join(d, "scene.bin")
        oracle_port.write_scene_bin(scene_file, photon_gpu.flatten_scene(s), spp,
                                    {"bneept": 0, "bvpt": 1, "bvptdl": 2}[s.estimator])
    out = subprocess.run([tool, scene_file, str(threads), str(scene.max_bounces), os.path.join(d, "out.rgbf32"),
                          str(repeats)], cwd=d, capture_output=True, text=True, check=True)
    records = []
    for line in out.stdout.splitlines():
        if not line.startswith("{"):
            continue
        r = json.loads(line)
        paths = per_spp_paths * spp
        records.append({
            "value": paths / r["render_s"] / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": kind, "paths": paths,
            "spp": spp, "render_s": r["render_s"],
            "sample": f"{scene.width}x{scene.height} x {spp} spp of the same scene ({paths} paths), "
                      f"{'phRender' if kind == 'reference' else 'oracle port render'} only "
                      f"({r['render_s']:.2f} s); scene load {r['load_s']:.1f} s and update "
                      f"{r['update_s']:.1f} s excluded"})
    return records


def roofline_of(kernel_ms: dict, rays: float, shadow_rays: float, iterations: float, counts: dict) -> dict:
    """HBM roofline of the kernel with the largest device time: algorithmic bytes (the traversal
    model from the counted nodes and triangles per ray) over its measured time, against the
    measured copy bandwidth; `traffic` is DRAM bytes per launch from the committed ncu capture,
    scaled by queue entries to this workload's average launch."""
    peaks = measured_peaks()
    nodes_per_ray = counts["nodes_closest"] / max(1.0, counts["rays"])
    tris_per_ray = counts["tris_closest"] / max(1.0, counts["rays"])
    s_nodes = counts["nodes_any"] / max(1.0, counts["shadow_rays"])
    s_tris = counts["tris_any"] / max(1.0, counts["shadow_rays"])
    # bytes per closest-hit ray: 32 ray in + 8 hit out + 80 per node + 48 per triangle
    bytes_closest = 40.0 + 80.0 * nodes_per_ray + 48.0 * tris_per_ray
    bytes_shadow = 48.0 + 80.0 * s_nodes + 48.0 * s_tris
    dominant = max(("extend_ms", "shadow_ms", "shade_ms"), key=lambda k: kernel_ms[k])
    # one trace launch serves both queues (the any-hit slot then only times two empty events)
    merged = kernel_ms["shadow_ms"] < 0.02 * kernel_ms["extend_ms"]
    if dominant == "shadow_ms":
        alg_bytes, kname = bytes_shadow * shadow_rays, "shadow (any hit)"
    elif dominant == "extend_ms" and merged:
        alg_bytes, kname = bytes_closest * rays + bytes_shadow * shadow_rays, "trace (closest + any hit)"
    elif dominant == "extend_ms":
        alg_bytes, kname = bytes_closest * rays, "extend (closest hit)"
    else:
        # shade: ray + hit + state in/out + triangle + shadow record per queued ray
        alg_bytes, kname = (32 + 8 + 80 + 48 + 112 + 48) * rays, "shade"
    achieved = alg_bytes / (kernel_ms[dominant] / 1e3) / 1e9
    traffic = None
    l2 = None
    prof_path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(prof_path):
        with open(prof_path) as f:
            rec = json.load(f).get(dominant) or {}
        entries = (shadow_rays if dominant == "shadow_ms" else
                   rays + shadow_rays if dominant == "extend_ms" and merged else rays) / max(1, iterations)
        if rec.get("dram_bytes_per_entry"):
            traffic = rec["dram_bytes_per_entry"] * entries
        if rec.get("l2_bytes_per_entry"):
            # the L2 side of the same kernel: bytes the SMs moved through L2 per launch (ncu
            # lts__t_bytes scaled by queue entries) over the kernel's measured time here, and
            # the L2 throughput fraction ncu reported for that launch
            l2_bytes = rec["l2_bytes_per_entry"] * entries
            launch_s = kernel_ms[dominant] / 1e3 / max(1, iterations)
            l2 = {"bytes_per_launch": l2_bytes, "achieved_gbs": l2_bytes / launch_s / 1e9,
                  "ncu_lts_throughput_pct": rec.get("lts_throughput_pct"),
                  "ncu_issue_active_pct": rec.get("issue_active_pct"),
                  "ncu_threads_per_instruction": rec.get("thread_inst_per_inst")}
    return {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "l2": l2,
            "algorithmic_bytes_per_launch": alg_bytes / max(1, iterations),
            "peak_source": peaks["source"],
            "model": {"bytes_per_closest_ray": bytes_closest, "nodes_per_closest_ray": nodes_per_ray,
                      "tris_per_closest_ray": tris_per_ray, "bytes_per_shadow_ray": bytes_shadow,
                      "nodes_per_shadow_ray": s_nodes, "tris_per_shadow_ray": s_tris}}


def rel_mse(x: np.ndarray, ref: np.ndarray, eps: float = 1e-2) -> float:
    """Mean over pixels and channels of (x - ref)^2 / (ref^2 + eps)."""
    return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref.astype(np.float64) ** 2 + eps)))


def guided_equal_time(num_boxes: int = 166_667, res: int = 256, ref_spp: int = 65536, probe_spp: int = 64,
                      target: float = 1e-3, warmup_renders: int = 8, warmup_spp: int = 32,
                      alpha: float = 0.5, depth: int = 1) -> dict:
    """Guided vs plain GPU BNEEPT on the slit-light room (2M triangles), as time to reach a relMSE
    target against a 65,536-spp plain render of the same scene.

    relMSE of an unbiased n-spp render falls as c/n, so each method is rendered once at a probe
    count, its relMSE gives the count that reaches `target`, and it is rendered again at that
    count: time_to_target = its device time x (its relMSE / target). The reference render is itself
    noisy: against it, an n-spp render measures c/n + c_plain/ref_spp, where the second term (the
    reference's own error, estimated from the plain renders) is the same for every method and is
    subtracted before the extrapolation. Guided renders start from a network trained by
    `warmup_renders` renders (training time reported apart) and keep training; `guided_frozen`
    renders with the trained network and no further training. alpha: the probability of sampling
    the learned mixture at a guided vertex; depth: the vertices guided, the first `depth` of each
    path (0: all). A ratio below 1 means guiding reaches the target
    sooner; the target is a ratio of at most 0.5.
    """
    import photon_gpu

    scene = scenes.slit_room(res, res, 1, 10, num_boxes=num_boxes)
    floor = {"relmse": 0.0}

    def to_target(rs, seed, plain=False):
        rs.clear()
        rs.render(probe_spp, max_bounces=10, seed=seed)
        e_probe = rel_mse(rs.film()[0], ref)
        if plain:
            # e = c/n + c/ref_spp for the plain estimator against its own reference
            floor["relmse"] = e_probe / (1.0 / probe_spp + 1.0 / ref_spp) / ref_spp
        c_probe = max(e_probe - floor["relmse"], 1e-12) * probe_spp
        spp = int(min(65536, max(probe_spp, np.ceil(c_probe / target))))
        rs.clear()
        r = rs.render(spp, max_bounces=10, seed=seed + 1)
        e = rel_mse(rs.film()[0], ref)
        if plain:
            floor["relmse"] = e / (1.0 / spp + 1.0 / ref_spp) / ref_spp
        e_own = max(e - floor["relmse"], 1e-12)
        return {"spp": spp, "ms": r["ms"], "relmse_vs_reference": e, "relmse": e_own, "probe_relmse": e_probe,
                "ms_to_target": r["ms"] * e_own / target}

    with photon_gpu.RenderScene(scene) as rs:
        t0 = time.time()
        rs.render(ref_spp, max_bounces=10, seed=1)
        ref = rs.film()[0]
        ref_s = time.time() - t0
        plain = to_target(rs, 100, plain=True)
        rs.set_guiding(True, True, alpha, 3e-3, 16384)
        rs.set_guiding_depth(depth)
        train_ms = 0.0
        for k in range(warmup_renders):
            rs.clear()
            train_ms += rs.render(warmup_spp, max_bounces=10, seed=200 + k)["ms"]
        guided = to_target(rs, 300)
        prof_guided = rs.profile(probe_spp, max_bounces=10, seed=310)
        info = rs.guide_info()
        rs.set_guiding(True, False, alpha, 3e-3, 16384)
        frozen = to_target(rs, 400)
        rs.set_guiding(False, False, alpha, 3e-3, 16384)
        prof_plain = rs.profile(probe_spp, max_bounces=10, seed=110)
    ratio = guided["ms_to_target"] / plain["ms_to_target"]
    return {
        "workload": f"slit_room {res}x{res}, {scene.num_tris} triangles, depth 10",
        "width": res, "height": res, "triangles": scene.num_tris, "max_bounces": 10,
        "reference_spp": ref_spp, "reference_s": ref_s, "target_relmse": target, "relmse_eps": 1e-2,
        "reference_noise_relmse": floor["relmse"], "alpha": alpha, "guided_depth": depth,
        "plain": plain, "guided": guided, "guided_frozen": frozen,
        "training": {"renders": warmup_renders, "spp": warmup_spp, "ms": train_ms, "final_loss": info["loss"]},
        # per-kernel device ms of one probe-spp render each (extend_ms: the merged trace launch)
        "cost_breakdown_ms": {"plain": prof_plain, "guided": prof_guided},
        "time_ratio": ratio,
        "time_ratio_with_training": (guided["ms_to_target"] + train_ms) / plain["ms_to_target"],
        "time_ratio_frozen": frozen["ms_to_target"] / plain["ms_to_target"],
    }


def c2_error(spp: int = 256) -> dict:
    """The error the benchmarked render carries: the 1M-triangle GGX scene at `spp` through the
    Photon C API at 64 x 64, against the reference CPU renderer's 65,536-spp render of the same
    scene (tests/golden/images.npz, made by tests/golden/make_golden_images.py). relMSE falls as
    1/spp, which gives the spp that reaches 1e-3."""
    import photon_gpu

    path = os.path.join(ROOT, "tests", "golden", "images.npz")
    if not os.path.exists(path):
        return {"unavailable": "tests/golden/images.npz missing"}
    d = np.load(path)
    if "c2_ggx1m_bneept" not in d:
        return {"unavailable": "no 65,536-spp reference render of the scene in images.npz"}
    ref = d["c2_ggx1m_bneept"]
    scene = scenes.ggx_sphere(level=8, width=64, height=64, spp=spp, max_bounces=10)
    with tempfile.TemporaryDirectory() as tmp:
        p2 = os.path.join(tmp, "scene.p2")
        with open(p2, "w") as f:
            f.write(scenes.to_sdl(scene, mesh_format="ply"))
        scenes.write_meshes(scene, tmp)
        scenes.write_env(scene, tmp)
        with photon_gpu.PhotonEngine() as eng:
            eng.set_working_directory(tmp)
            assert eng.load_file(p2), eng.errors()
            eng.set_max_bounces(scene.max_bounces)
            eng.set_seed(11)
            eng.update()
            eng.render()
            img = eng.frame()
    err = rel_mse(img, ref)
    return {"spp": spp, "relmse": err, "spp_for_relmse_1e-3": int(np.ceil(spp * err / 1e-3)),
            "reference": f"reference CPU renderer, {int(d['c2_ggx1m_bneept__spp'])} spp", "resolution": "64x64",
            "mean_ratio": (img.mean(axis=(0, 1)) / ref.mean(axis=(0, 1))).tolist(), "eps": 1e-2}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload in FLAT_WORKLOADS:
        scene_list = FLAT_WORKLOADS[args.workload]()
        rec = cpu_sample_many(scene_list, args.cpu_seconds, PORT_PATHS_PER_CORE_S[args.workload])
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": rec["value"], "unit": "Mpaths/s",
            "n_gpus": args.gpus, "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes)",
            "config": {"workload": args.workload, "scenes": len(scene_list),
                       "triangles": int(sum(sc.num_tris for sc in scene_list))},
            "cpu_baseline": rec,
            "e2e": {"value": rec["value"], "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    scene = workload(args.workload)
    with tempfile.TemporaryDirectory() as tmp:
        samples = cpu_sample(scene, tmp, target_seconds=args.cpu_seconds, repeats=args.warmup + args.steps)
        timed = samples[args.warmup:] if len(samples) > args.warmup else samples
        vals = [s["value"] for s in timed if s["value"]]
        value = statistics.median(vals) if vals else None
        base = timed[-1]
        # A step is one render of the bounded sample (the same scene at base["spp"] samples per
        # pixel), timed around phRender; the full frame's time is extrapolated from the rate and
        # reported under its own key.
        sample_ms = [1e3 * s["render_s"] for s in timed if s.get("render_s")]
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpaths/s",
            "n_gpus": args.gpus, "steps": len(timed), "warmup": len(samples) - len(timed),
            "ms_per_step": statistics.median(sample_ms) if sample_ms else None,
            "ms_per_full_frame_extrapolated":
                (scene.width * scene.height * scene.spp / (value * 1e6) * 1e3) if value else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": args.workload, "width": scene.width, "height": scene.height,
                       "spp": scene.spp, "max_bounces": scene.max_bounces, "triangles": scene.num_tris,
                       "step": f"one render of {base.get('spp')} spp (bounded sample of the {scene.spp}-spp frame)"},
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": base["cores"], "kind": base["kind"],
                             "sample": base["sample"]},
            "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))


def run_ours(args) -> None:
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local_rank))
        dist = dist_mod

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    import photon_gpu

    photon_gpu.load()
    scene = workload(args.workload)
    if args.spp:
        scene.spp = args.spp
    paths_per_step = scene.width * scene.height * scene.spp
    l2_flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2

    with tempfile.TemporaryDirectory() as tmp:
        p2 = write_scene(scene, tmp)
        eng = photon_gpu.PhotonEngine()
        eng.set_working_directory(tmp)
        t0 = time.time()
        assert eng.load_file(p2), eng.errors()
        load_s = time.time() - t0
        eng.set_max_bounces(scene.max_bounces)
        eng.set_seed(1000003 * rank + 7)
        eng.update()
        update_s = eng.info()["update_seconds"]
        # launch shapes picked for this scene by the autotuner (untimed calibration renders)
        tuned = eng.autotune(rebuild=True) if args.autotune else None

        for _ in range(args.warmup):
            eng.clear_film()
            eng.render()

        # Traversal counts (untimed): nodes / triangles per ray for the algorithmic-bytes model.
        counts = eng.profile(2, 4)
        # Per-kernel device times with CUDA events around each launch (untimed pass).
        kprof = eng.profile(1, scene.spp)

        # ---- timed region: device time of K full renders
        barrier()
        with ClockSampler(local_rank) as clocks:
            device_ms = 0.0
            launches = 0
            wall0 = time.time()
            for _ in range(args.steps):
                l2_flush.fill_(1.0)
                torch.cuda.synchronize()
                eng.clear_film()
                eng.render()
                info = eng.info()
                assert info["paths"] == paths_per_step
                device_ms += info["device_ms"]
                launches += eng.launch_count()
            wall = time.time() - wall0
        barrier()
        device_ms = max_over_ranks(device_ms)
        value = world * paths_per_step * args.steps / (device_ms / 1e3) / 1e6

        # ---- end to end through the public C API, frame copied to host every step
        barrier()
        e2e_s = 0.0
        for _ in range(args.steps):
            eng.clear_film()
            t = time.time()
            eng.render()
            frame = eng.frame()
            e2e_s += time.time() - t
        barrier()
        e2e_s = max_over_ranks(e2e_s)
        e2e_value = world * paths_per_step * args.steps / e2e_s / 1e6
        d2h = int(scene.width * scene.height * 3 * 4)   # the frame developed on the GPU (float32 RGB) read back
        mean_rgb = frame.reshape(-1, 3).mean(0).tolist()
        eng.close()

        # ---- roofline of the dominant kernel
        kernel_ms = {k: kprof[k] for k in ("prepare_ms", "regen_ms", "extend_ms", "shade_ms", "shadow_ms")}
        total_k = sum(kernel_ms.values())
        rays = kprof["rays"]
        shadow_rays = kprof["shadow_rays"]
        roofline = roofline_of(kernel_ms, rays, shadow_rays, kprof["iterations"], counts)

    clock = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": device_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": args.workload, "width": scene.width, "height": scene.height, "spp": scene.spp,
                   "max_bounces": scene.max_bounces, "triangles": scene.num_tris, "estimator": "bneept",
                   "l2": "256 MiB write between timed steps", "parallelism": f"replicas x{world}",
                   "tuned": tuned},
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
                "path": "phRender + phAquireFrameRaw + phGetFrameRgbData (scene resident after phUpdate)"},
        "gpu_launches": launches,
        "roofline": roofline,
        "kernel_ms_per_step": {k: v for k, v in kernel_ms.items()},
        "kernel_share": {k: v / total_k for k, v in kernel_ms.items()},
        "rays_per_step": {"closest": rays, "shadow": shadow_rays},
        "mrays_per_s": (rays + shadow_rays) / (device_ms / args.steps / 1e3) / 1e6,
        "clocks": {"sm_mhz": clock["sm_mhz"], "sm_max_mhz": clock["sm_max_mhz"], "reasons": clock["reasons"]},
        "host": {"scene_load_s": load_s, "update_s": update_s, "wall_s_timed": wall, "image_mean_rgb": mean_rgb},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as tmp:
            line["cpu_baseline"] = cpu_sample(scene, tmp, target_seconds=args.cpu_seconds)[-1]
    if rank == 0 and world == 1 and args.workload == "ggx_1m":
        line["error_vs_65536spp"] = c2_error(scene.spp)
        if not args.no_other_workloads:
            line["other_workloads"] = other_workloads()
    if rank == 0 and world == 1 and not args.no_guided:
        line["guided_equal_time"] = guided_equal_time()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


# Workloads too large for SDL text (the SDL vector3-array is text only): built and rendered
# through the flat scene ABI (pgpu_scene_create / pgpu_scene_render), one RenderScene each.
FLAT_WORKLOADS = {
    # many-light city: 447^2 lognormal buildings, 21.6M triangles, 10,000 lights, 1920x1080, 1024 spp
    "city": lambda: [scenes.city()],
    # 64 seeded scenes, 1k-500k triangles, 128^2-1024^2, 16-256 spp, rendered one after another
    "batched": lambda: [scenes.batch_scene(i) for i in range(64)],
    # the learned-guiding room rendered plain: 2M triangles, one light behind a slit, 1024^2, 64 spp
    "slit_room": lambda: [scenes.slit_room()],
}
# The oracle port's cost on these workloads (Mpaths/s per host thread, measured on the GPU box's
# 16 threads); only used to size the bounded CPU sample, the reported rate is always measured.
PORT_PATHS_PER_CORE_S = {"city": 0.054e6, "batched": 0.10e6, "slit_room": 0.012e6}


def run_flat(args) -> None:
    """One step = every scene of the workload rendered once with its own spp (device time summed);
    e2e adds each developed frame's copy to host memory."""
    import torch

    import photon_gpu

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    photon_gpu.load()
    t0 = time.time()
    scene_list = FLAT_WORKLOADS[args.workload]()
    gen_s = time.time() - t0
    if args.spp:
        for sc in scene_list:
            sc.spp = args.spp
    t0 = time.time()
    rss = [photon_gpu.RenderScene(sc, builder=args.builder) for sc in scene_list]
    build_s = time.time() - t0
    tuned = None
    if args.autotune and len(rss) > 1 and args.batch_mode == "wavefront":
        # launch shapes of the one-wavefront render (untimed calibration wavefronts)
        tuned = [photon_gpu.autotune_wavefront(rss, [sc.spp for sc in scene_list],
                                               max_bounces=scene_list[0].max_bounces)]
    elif args.autotune:
        # launch shapes per scene (untimed calibration renders; the leaf-size rebuild only for
        # single-scene workloads)
        tuned = [rs.autotune(sc.spp, max_bounces=sc.max_bounces, rebuild=len(rss) == 1)
                 for sc, rs in zip(scene_list, rss)]
    paths_per_step = sum(sc.width * sc.height * sc.spp for sc in scene_list)
    l2_flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2
    seed = 1000003 * rank + 7

    def one_pass(read_back: bool = False):
        ms, launches = 0.0, 0
        if args.batch_mode == "wavefront" and len(scene_list) > 1:
            # every scene in one wavefront: one path pool, one launch per kernel per iteration
            for rs in rss:
                rs.clear()
            ms = photon_gpu.render_scenes_wavefront(rss, [sc.spp for sc in scene_list],
                                                    max_bounces=scene_list[0].max_bounces, seed=seed)
            launches = rss[0].launches()
            if read_back:
                for rs in rss:
                    rs.film(with_sums=False)
            return ms, launches
        if args.batch_mode == "streams" and args.concurrency > 1 and len(scene_list) > 1:
            # all scenes of the step at once, `concurrency` of them in flight on their own streams;
            # the step's time is the batch's span
            for rs in rss:
                rs.clear()
            ms = photon_gpu.render_scenes(rss, [sc.spp for sc in scene_list], max_bounces=scene_list[0].max_bounces,
                                          seed=seed, concurrency=args.concurrency)
            launches = sum(rs.launches() for rs in rss)
            if read_back:
                for rs in rss:
                    rs.film(with_sums=False)
            return ms, launches
        for sc, rs in zip(scene_list, rss):
            rs.clear()
            ms += rs.render(sc.spp, max_bounces=sc.max_bounces, seed=seed)["ms"]
            launches += rs.launches()
            if read_back:
                rs.film(with_sums=False)
        return ms, launches

    for _ in range(args.warmup):
        one_pass()
    torch.cuda.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        device_ms, launches = 0.0, 0
        wall0 = time.time()
        for _ in range(args.steps):
            l2_flush.fill_(1.0)
            torch.cuda.synchronize()
            ms, n = one_pass()
            device_ms += ms
            launches += n
        wall = time.time() - wall0
    value = paths_per_step * args.steps / (device_ms / 1e3) / 1e6
    e2e_s = 0.0
    for _ in range(args.steps):
        t = time.time()
        one_pass(read_back=True)
        e2e_s += time.time() - t
    e2e_value = paths_per_step * args.steps / e2e_s / 1e6
    d2h = sum(sc.width * sc.height * 3 * 4 for sc in scene_list)

    # per-kernel device time (events around every launch) and traversal counts, untimed
    kernel_ms = dict.fromkeys(("prepare_ms", "regen_ms", "extend_ms", "shade_ms", "shadow_ms"), 0.0)
    counts = dict.fromkeys(("rays", "shadow_rays", "nodes_closest", "tris_closest", "nodes_any", "tris_any"), 0)
    rays = shadow_rays = iterations = 0
    for sc, rs in zip(scene_list, rss):
        prof = rs.profile(sc.spp, max_bounces=sc.max_bounces, seed=seed)
        for k in kernel_ms:
            kernel_ms[k] += prof[k]
        full = rs.count(sc.spp, max_bounces=sc.max_bounces, seed=seed)
        rays += full["rays"]
        shadow_rays += full["shadow_rays"]
        iterations += full["iterations"]
        for k in counts:
            counts[k] += full[k]
    for rs in rss:
        rs.close()
    total_k = sum(kernel_ms.values())
    clock = clocks.summary()
    spps = sorted({sc.spp for sc in scene_list})
    line = {
        "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": device_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes)",
        "config": {"workload": args.workload, "scenes": len(scene_list),
                   "triangles": int(sum(sc.num_tris for sc in scene_list)), "paths_per_step": paths_per_step,
                   "resolution": sorted({f"{sc.width}x{sc.height}" for sc in scene_list})[:4],
                   "spp": spps if len(spps) <= 4 else [spps[0], spps[-1]],
                   "max_bounces": scene_list[0].max_bounces, "estimator": "bneept", "bvh": args.builder,
                   "batch_mode": args.batch_mode if len(scene_list) > 1 else "single",
                   "concurrency": args.concurrency if len(scene_list) > 1 and args.batch_mode == "streams" else 1,
                   "l2": "256 MiB write between timed steps", "parallelism": f"replicas x{world}",
                   "tuned": (tuned[0] if tuned and len(tuned) == 1 else
                             {"scenes": len(tuned), "ms_default": sum(t["ms_default"] for t in tuned),
                              "ms_tuned": sum(t["ms_tuned"] for t in tuned),
                              "shapes": sorted({(t["capacity"], t["refill"], t["blocks_per_sm"], t["leaf_tris"])
                                                for t in tuned})} if tuned else None)},
        "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
                "path": "pgpu_scene_render + pgpu_scene_film (frame developed on the GPU, copied to host)"},
        "gpu_launches": launches,
        "roofline": roofline_of(kernel_ms, rays, shadow_rays, iterations, counts),
        "kernel_ms_per_step": kernel_ms,
        "kernel_share": {k: v / total_k for k, v in kernel_ms.items()},
        "rays_per_step": {"closest": rays, "shadow": shadow_rays},
        "mrays_per_s": (rays + shadow_rays) / (device_ms / args.steps / 1e3) / 1e6,
        "clocks": {"sm_mhz": clock["sm_mhz"], "sm_max_mhz": clock["sm_max_mhz"], "reasons": clock["reasons"]},
        "host": {"scene_generation_s": gen_s, "bvh_build_and_upload_s": build_s, "wall_s_timed": wall},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample_many(scene_list, args.cpu_seconds, PORT_PATHS_PER_CORE_S[args.workload])
    if rank == 0:
        print(json.dumps(line))


def other_workloads(steps: int = 2, scale: int = 8) -> dict:
    """The other benchmarked configurations measured in the same run, each at 1/scale of its
    samples per pixel (at least 8): the batched 64 scenes as one wavefront, the slit-light room
    rendered plain, and the many-light city. Device-timed Mpaths/s over `steps` renders after one
    warm-up render (launch shapes autotuned first, untimed)."""
    import torch

    import photon_gpu

    out = {}
    l2_flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for name in ("batched", "slit_room", "city"):
        t0 = time.time()
        scene_list = FLAT_WORKLOADS[name]()
        for sc in scene_list:
            sc.spp = max(8, sc.spp // scale)
        rss = [photon_gpu.RenderScene(sc) for sc in scene_list]
        setup_s = time.time() - t0
        spp = [sc.spp for sc in scene_list]
        bounces = scene_list[0].max_bounces
        if len(rss) > 1:
            tuned = photon_gpu.autotune_wavefront(rss, spp, max_bounces=bounces)
            render = lambda: photon_gpu.render_scenes_wavefront(rss, spp, max_bounces=bounces, seed=7)
        else:
            tuned = rss[0].autotune(spp[0], max_bounces=bounces, rebuild=True)
            render = lambda: rss[0].render(spp[0], max_bounces=bounces, seed=7)["ms"]
        paths = sum(sc.width * sc.height * sc.spp for sc in scene_list)
        for rs in rss:
            rs.clear()
        render()
        ms = 0.0
        for _ in range(steps):
            l2_flush.fill_(1.0)
            torch.cuda.synchronize()
            for rs in rss:
                rs.clear()
            ms += render()
        out[name] = {"value": paths * steps / (ms / 1e3) / 1e6, "unit": "Mpaths/s", "steps": steps,
                     "paths_per_step": paths, "ms_per_step": ms / steps, "scenes": len(scene_list),
                     "triangles": int(sum(sc.num_tris for sc in scene_list)),
                     "spp": sorted(set(spp)) if len(set(spp)) <= 2 else [min(spp), max(spp)],
                     "spp_scale": f"1/{scale} of the configuration's spp (at least 8)",
                     "mode": "one wavefront" if len(rss) > 1 else "single scene",
                     "tuned": {k: tuned[k] for k in ("capacity", "refill", "blocks_per_sm", "leaf_tris",
                                                     "ms_default", "ms_tuned")},
                     "setup_s": setup_s}
        for rs in rss:
            rs.close()
    return out


def cpu_sample_many(scene_list, target_seconds: float, paths_per_core_s: float = EST_CPU_PATHS_PER_CORE_S) -> dict:
    """CPU baseline of a multi-scene or very large workload: the oracle port (binary scene file;
    SDL text of tens of millions of triangles is impractical to parse) on the first scenes, each
    with spp reduced to a bounded sample, paths summed over render time."""
    picked = scene_list[:4]
    paths = secs = 0.0
    cores, kinds = os.cpu_count() or 1, set()
    with tempfile.TemporaryDirectory() as tmp:
        for sc in picked:
            rec = cpu_sample(sc, tmp, target_seconds=target_seconds / len(picked), force_port=True,
                             paths_per_core_s=paths_per_core_s)[-1]
            if not rec["value"]:
                return rec
            n = rec["paths"]
            paths += n
            secs += n / (rec["value"] * 1e6)
            kinds.add(rec["kind"])
    return {"value": paths / secs / 1e6, "unit": "Mpaths/s", "cores": cores, "kind": "/".join(sorted(kinds)),
            "sample": f"{len(picked)} of {len(scene_list)} scenes at reduced spp ({int(paths)} paths, "
                      f"{secs:.1f} s of render time; BVH build excluded)"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ggx_1m")
    ap.add_argument("--spp", type=int, default=0, help="override samples per pixel")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-guided", action="store_true", help="skip the guided-vs-plain equal-time comparison")
    ap.add_argument("--builder", default="sah", choices=["sah", "gpu"], help="BVH builder of flat workloads")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="skip the reduced-spp measurement of the batched, slit-room and city workloads")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="render with the fixed default launch shapes instead of autotuned ones")
    ap.add_argument("--batch-mode", default="wavefront", choices=["wavefront", "streams", "serial"],
                    help="multi-scene workloads: one wavefront for all scenes, scenes on concurrent streams, "
                         "or one after another")
    ap.add_argument("--concurrency", type=int, default=4,
                    help="scenes of a multi-scene workload rendered at once (1: one after another)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in FLAT_WORKLOADS:
        run_flat(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
