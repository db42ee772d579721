"""Benchmark of the Conditional ReSTIR PT frame loop (one step = one frame).

Workload: the large configuration -- 1920x1080 on a room of 64 displaced
icospheres (5 subdivisions, 20,480 triangles each, 1,310,988 triangles in
total with the room and the 256 emissive triangles), max depth 8, prefix
length 2, prefix-endpoint search k = 8, 1 temporal + 2 spatial suffix passes
of 5 neighbours, FP32 reservoirs, a 60-frame camera orbit, seed 1.

Metric: resampled paths per second (25 per pixel per frame: prefix temporal
2 + suffix temporal 2 + suffix spatial 2 x (5 + 1) + final gather 8 + 1) and
ms per frame.  `value` is measured with everything resident on the device;
`e2e` goes through the C ABI with the frame's camera in and the image copied
out to pinned host memory every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl crisb|reference]

Under torchrun each rank renders its own view of the orbit (weak scaling, no
collective on the data path); the reported time is the max over ranks.
"""
from __future__ import annotations

import argparse
import copy
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PATHS_PER_PIXEL_LARGE = 25  # 2 + 2 + 2 * (5 + 1) + (8 + 1)
METRIC = "1080p ms/frame & paths/s at fixed relMSE; batched+adjoint vs plain, same GPU"
UNIT = "resampled paths/s"


def workload(name: str):
    from crisoptix_b200 import scenes

    if name == "large":
        desc, cam = scenes.sphere_room(num_spheres=64, subdiv=5, num_emitters=256, seed=1)
        return desc, cam, 1920, 1080, PATHS_PER_PIXEL_LARGE
    if name == "small":
        desc, cam = scenes.cornell_box()
        return desc, cam, 256, 256, 2 + 2 + (3 + 1) + 1
    raise ValueError(name)


def params_for(name: str, scene_size: float):
    from crisoptix_b200 import _abi
    from crisoptix_b200.scenes import Camera  # noqa: F401

    p = _abi.Params()
    base = dict(renderer_type=_abi.CONDITIONAL_RESTIR, nee_prob=0.3, max_path_len=8, enable_accum=0,
                recon_min_distance=0.01 * scene_size, recon_min_roughness=0.2, prefix_len=2, prefix_enable_temporal=1,
                prefix_enable_spatial=0, prefix_spatial_count=1, prefix_spatial_rounds=1, suffix_enable_temporal=1,
                suffix_enable_spatial=1, suffix_spatial_count=5, suffix_spatial_rounds=2, gather_n=1, gather_m=9,
                gather_radius=0.01, gather_radius_type=_abi.RADIUS_PATH_LENGTH, window_radius=10,
                storage=_abi.STORAGE_FP32, seed=1)
    if name == "small":
        base.update(max_path_len=4, prefix_len=1, suffix_spatial_count=3, suffix_spatial_rounds=1, gather_m=1,
                    window_radius=30, seed=0)
    for k, v in base.items():
        setattr(p, k, v)
    return p


def config_for(name: str, W: int, H: int, n_tris: int, p, ppp: int, world: int, graph: bool = True) -> dict:
    """The `config` object of both arms' JSON lines."""
    return {"workload": f"{name}: {W}x{H} conditional ReSTIR PT, {n_tris} triangles, k={p.gather_m - 1}, "
                        f"{p.suffix_spatial_rounds}x{p.suffix_spatial_count} spatial, max depth {p.max_path_len}, "
                        f"{'FP16' if p.storage == 1 else 'FP32'} storage"
                        + (", reprojected temporal reuse" if p.motion_mode == 2 else ""),
            "paths_per_pixel": ppp, "l2": "working set (reservoirs, BVH) larger than L2",
            "parallelism": f"view-sharded replicas x{world}", "frame_as_cuda_graph": graph}


# Compulsory bytes per pixel per frame of the resampling kernels (the
# bandwidth-bound part of each reuse pass: MIS weights and reservoir
# streaming over records and shift results).  Every record a kernel touches
# is counted once per kernel (a neighbour's reservoir is another pixel's own
# record), at nominal occupancy: all k / spatial neighbours present.
# Records: prefix reservoir 144 B (FP32) / 80 B (FP16 storage), canonical
# prefix 128 B, suffix reservoir 112 B / 64 B, canonical suffix 112 B,
# G-buffer RNG 8 B, shift result 16 B.
def resample_bytes(k: int, spatial_count: int, spatial_rounds: int, copy_prefix_back: bool,
                   fp16: bool = False) -> dict:
    pr, sr = (80, 64) if fp16 else (144, 112)
    prefix_combine = pr + 128 + pr + 8 + 8 + 4 + 2 * 16 + pr + (pr if copy_prefix_back else 0)
    temporal_combine = sr + 112 + 8 + 8 + 4 + 2 * 16 + sr
    spatial_select = 3 * 4 + 8 + 8 + 4 * spatial_count + 8
    spatial_combine = sr + 8 + 8 + 8 + 4 * spatial_count + 2 * 16 * spatial_count + sr
    gather_combine = 12 + 12 + 32 + 8 * k + 20 + 2 * 16 * k + 12
    return {"prefix_combine": prefix_combine, "temporal_combine": temporal_combine,
            "spatial_select": spatial_rounds * spatial_select, "spatial_combine": spatial_rounds * spatial_combine,
            "gather_combine": gather_combine}


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the seven
# resampling launches of one frame, from ncu captures of the large workload
# at 960x540 (518,400 px, caches flushed before each launch), per reservoir
# storage, with the pixel count it was taken at; scaled by pixels to the bench
# resolution.
PROFILED_TRAFFIC = {"resampling": (469.79e6, 960 * 540), "resampling_fp16": (333.55e6, 960 * 540)}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def tonemap_timing(frame, W: int, H: int, stream, stack: int = 16, reps: int = 10) -> dict:
    """crisb_tonemap_srgb8 on `stack` copies of the rendered frame (inputs
    larger than L2), 12 bytes read and 3 written per pixel."""
    import torch

    from crisoptix_b200 import image

    src = frame.view(1, H * W * 3).repeat(stack, 1).contiguous()
    dst = torch.empty(src.shape, dtype=torch.uint8, device=src.device)
    sptr = stream.cuda_stream
    for _ in range(3):
        image.tonemap(src.view(-1, 3), dst.view(-1, 3), sptr)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        image.tonemap(src.view(-1, 3), dst.view(-1, 3), sptr)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    px = stack * W * H
    peak, kind = measured_peaks()
    gbs = 15.0 * px / (ms / 1000.0) / 1e9
    return {"kernel": "k_tonemap_srgb8", "pixels_per_launch": px, "frames_per_launch": stack,
            "bytes_per_pixel": 15, "ms_per_launch": ms, "ms_per_frame": ms / stack, "achieved_gbs": gbs,
            "frac": gbs / peak, "peak_kind": f"{kind} copy bandwidth"}


def cpu_baseline(desc, cam, name: str, threads: int, frames: int, warm: int = 1, scale: int = 4):
    """The oracle (a host port of the reference's device code) on a bounded
    sample: the same scene and parameters at 1/scale of the resolution."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as op
    from crisoptix_b200 import scenes

    _, _, W, H, ppp = workload(name)
    w, h = max(W // scale, 8), max(H // scale, 8)
    op.set_threads(threads)
    o = op.Oracle.from_scene(desc, w, h, params_for(name, 0.0))
    p = params_for(name, o.scene_size)
    o.set_params(p)
    out = np.zeros((h, w, 3), np.float32)
    for f in range(warm):
        o.render_frame(scenes.orbit_camera(cam, f, 60), out)
    t0 = time.perf_counter()
    for f in range(frames):
        o.render_frame(scenes.orbit_camera(cam, warm + f, 60), out)
    dt = time.perf_counter() - t0
    return {"value": ppp * w * h * frames / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{w}x{h} (1/{scale * scale} of the pixels) of the same scene and parameters, "
                      f"{frames} frame(s) after {warm} warm-up frame(s), {threads} OpenMP threads",
            "ms_per_frame": 1000.0 * dt / frames}


def run_reference(args):
    """--impl reference: the oracle port of the reference's device code on the
    host cores (the reference itself needs OptiX and cannot run here)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # the multiview workload renders the large scene: its reference sample is
    # the large workload's
    name = "large" if args.workload == "multiview" else args.workload
    desc, cam, W, H, ppp = workload(name)
    threads = os.cpu_count() or 1
    # K timed steps after W warm-up steps, each one frame of the orbit on the
    # bounded sample (1/cpu_scale^2 of the pixels; about a second per frame
    # on 16 host cores)
    cb = cpu_baseline(desc, cam, name, threads, args.steps, warm=args.warmup, scale=args.cpu_scale)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["ms_per_frame"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_for(name, W, H, desc.num_world_triangles, params_for(name, 1.0), ppp, args.gpus),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CrisOptix needs the OptiX SDK and an OpenGL window; its CPU-side stand-in is the oracle port "
                    "of its device code"}
    print(json.dumps(line), flush=True)


def comparison_arms(sc, cam, W: int, H: int, p, ppp: int, value: float, ms_per_frame: float, args) -> dict:
    """The comparison the benchmark metric names, measured on the same GPU
    right after the main loop:
      - single view: FP32 storage (the main `value`) and FP16 storage, each
        with the relMSE of orbit frame 30 against one FP64-accumulated
        path-traced reference of that frame (`arm_ref_spp` samples per pixel,
        fewer than the 4096 of the full quality run, to stay within the
        benchmark's time; stated in the line), beside the plain path tracer
        at equal time (the samples of frame 30's camera that fit in one FP32
        ReSTIR frame's time) and the FP32 form with reprojected temporal
        reuse, scored against the same reference;
      - 16 uneven views: the plain form (FP32 storage, views one after another)
        against the batched form (FP16 storage, one CUDA graph per frame with
        a branch per view), and their ratio of resampled paths/s;
      - the path-replay adjoint of the resampled estimator on the same
        workload: one backward pass (dLoss/dimage = 1 everywhere) and one
        evaluation of the frozen estimator, beside the frame time."""
    import torch

    from crisoptix_b200 import Renderer, _abi, quality, scenes

    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    q = copy.copy(p)
    q.storage = _abi.STORAGE_FP16
    r16 = Renderer(W, H, sc, q)
    out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    cams = [scenes.orbit_camera(cam, f, 60) for f in range(60)]
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            r16.launch_frame(cams[i], out.data_ptr(), sptr)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the frames of the orbit the main (FP32) loop timed: early frames cost
    # more than later ones, so both arms average the same stretch
    arm_steps = args.arm_steps or args.steps
    a.record(stream)
    for i in range(arm_steps):
        r16.launch_frame(cams[(args.warmup + i) % 60], out.data_ptr(), sptr)
    b.record(stream)
    torch.cuda.synchronize()
    r16.check_device_errors()
    ms16 = a.elapsed_time(b) / arm_steps
    del r16
    cam_of = lambda f: scenes.orbit_camera(cam, f, 60)  # noqa: E731
    ref = quality.reference_image(sc, W, H, cam_of(30), p, args.arm_ref_spp)
    q32 = quality.score(sc, W, H, cam_of, p, 31, args.arm_ref_spp, ref=ref)
    q16 = quality.score(sc, W, H, cam_of, q, 31, args.arm_ref_spp, ref=ref)
    qpt = quality.pt_equal_time(sc, W, H, cam_of(30), p, ms_per_frame, ref)
    qrp = copy.copy(p)
    qrp.motion_mode = _abi.MOTION_REPROJECT
    q32rp = quality.score(sc, W, H, cam_of, qrp, 31, args.arm_ref_spp, ref=ref)
    adj = adjoint_time(sc, cam, W, H, p, args.warmup, 3)
    mv_plain = multiview_time(_abi.STORAGE_FP32, False, args.arm_mv_steps, 2)
    mv_batch = multiview_time(_abi.STORAGE_FP16, True, args.arm_mv_steps, 2)
    keep = ("relmse", "relmse_trimmed_0.1pct")
    return {
        "single_view_fp32": {"value": value, "ms_per_frame": ms_per_frame,
                             "relmse": {k: q32[k] for k in keep}},
        "single_view_fp16": {"value": ppp * W * H * 1000.0 / ms16, "ms_per_frame": ms16, "steps": arm_steps,
                             "relmse": {k: q16[k] for k in keep}},
        "fp16_over_fp32": ms_per_frame / ms16,
        "relmse_reference": {"kind": "path tracer (TraceCompletePath), FP64 accumulation", "spp": args.arm_ref_spp,
                             "frame": 30},
        "single_view_fp32_reprojected": {"relmse": {k: q32rp[k] for k in keep},
                                         "note": "temporal reuse from the primary hit reprojected into the previous "
                                                 "camera (CRISB_MOTION_REPROJECT) instead of the same pixel"},
        "plain_pt_equal_time": {"equal_time_spp": qpt["equal_time_spp"], "ms_per_spp": qpt["ms_per_spp"],
                                "relmse_by_spp": qpt["scores"],
                                "note": "the path tracer at frame 30's camera, one sample per frame, scored at "
                                        "the whole sample counts either side of one ReSTIR FP32 frame's time; "
                                        "its own random stream"},
        "multiview_plain_fp32": dict(mv_plain, steps=args.arm_mv_steps),
        "multiview_batched_fp16": dict(mv_batch, steps=args.arm_mv_steps),
        "batched_fp16_over_plain_fp32": mv_batch["value"] / mv_plain["value"],
        "adjoint_fp32": adj,
        "unit": UNIT,
    }


def run_crisb(args):
    import torch

    from crisoptix_b200 import Renderer, Scene, _abi, scenes, sharding

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    desc, cam, W, H, ppp = workload(args.workload)
    if args.res:
        W, H = (int(v) for v in args.res.lower().split("x"))
    sc = Scene(desc)
    p = params_for(args.workload, sc.scene_size)
    p.storage = _abi.STORAGE_FP16 if args.storage == "fp16" else _abi.STORAGE_FP32
    p.motion_mode = _abi.MOTION_REPROJECT if args.motion == "reproject" else _abi.MOTION_NONE
    free0 = torch.cuda.mem_get_info()[0]
    r = Renderer(W, H, sc, p)
    torch.cuda.synchronize()
    renderer_bytes = free0 - torch.cuda.mem_get_info()[0]
    r.set_graph(not args.no_graph)
    tuned = r.autotune(cam, 3) if args.autotune else None
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    offset = sharding.orbit_offset(rank, world)  # each rank renders its own view of the orbit
    n_frames = args.warmup + args.steps
    cams = [scenes.orbit_camera(cam, offset + f, 60) for f in range(2 * n_frames + 8)]

    def frame(i):
        r.launch_frame(cams[i % len(cams)], out.data_ptr(), sptr)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            frame(i)
    torch.cuda.synchronize()
    r.check_device_errors()

    # ---- device-resident timing ------------------------------------------------
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        frame(args.warmup + i)
    t_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    launches_per_frame = r.stats()["kernel_launches"]
    ms = sharding.max_over_ranks(t_start.elapsed_time(t_end), dist, "cuda")
    ms_per_frame = ms / args.steps
    value = sharding.whole_job_rate(ppp * W * H, args.steps, world, ms)

    # ---- per-pass and per-kernel-class breakdown (CUDA events on the stream) ----
    r.set_timing(1)
    keys = ("prefix_gen_temp_ms", "prefix_spatial_ms", "suffix_gen_temp_ms", "suffix_spatial_ms", "prefix_store_ms",
            "final_gather_ms", "total_ms", "trace_ms", "shift_ms", "resample_ms", "search_ms", "shade_ms", "other_ms")
    passes = {k: 0.0 for k in keys}
    n_pass = 3
    for i in range(n_pass):
        frame(args.warmup + i)
        st = r.stats()
        for k in keys:
            passes[k] += st[k] / n_pass
    r.set_timing(2)  # ray counters (statistics only: adds atomics to the traversal)
    frame(args.warmup)
    rays = r.stats()
    r.set_timing(0)
    r.check_device_errors()

    # ---- end to end through the C ABI with host buffers ------------------------
    # Two output buffers: frame i's device-to-host copy (pinned host memory,
    # its own stream) overlaps frame i + 1, and a frame waits for the copy
    # that last read its buffer.  Every frame's copy is inside the timed region.
    outs = [out, torch.zeros_like(out)]
    hosts = [torch.empty(W * H * 3, dtype=torch.float32, pin_memory=True) for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [None, None]
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_steps = args.steps  # the same frames of the orbit as the device-resident loop
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e_start.record(stream)
    for i in range(e_steps):
        j = i % 2
        if copied[j] is not None:
            stream.wait_event(copied[j])
        r.launch_frame(cams[(args.warmup + i) % len(cams)], outs[j].data_ptr(), sptr)
        rendered = torch.cuda.Event()
        rendered.record(stream)
        copy_stream.wait_event(rendered)
        with torch.cuda.stream(copy_stream):
            hosts[j].copy_(outs[j], non_blocking=True)
        copied[j] = torch.cuda.Event()
        copied[j].record(copy_stream)
    stream.wait_stream(copy_stream)
    e_end.record(stream)
    torch.cuda.synchronize()
    host = hosts[(e_steps - 1) % 2]
    e_ms = sharding.max_over_ranks(e_start.elapsed_time(e_end), dist, "cuda")
    e2e_value = sharding.whole_job_rate(ppp * W * H, e_steps, world, e_ms)
    img_mean = float(host.mean())
    tone = tonemap_timing(out, W, H, stream)

    # ---- the comparison arms the metric names (same box, same run) ------------
    arms = None
    if not args.no_arms and world == 1 and args.workload == "large" and not args.res:
        arms = comparison_arms(sc, cam, W, H, p, ppp, value, ms_per_frame, args)

    # ---- roofline of the resampling kernels; traversal in rays/s -----------------
    peak, peak_kind = measured_peaks()
    # algorithmic bytes: what the resampling kernels read and write for the
    # work present in this frame (valid neighbours, chosen records), counted
    # on the device at statistics level 2 (crisb_stats.resample_bytes)
    tally = rays["resample_bytes"]
    res_bytes = sum(tally.values())
    achieved = res_bytes / (passes["resample_ms"] / 1000.0) / 1e9
    traffic = None
    key = "resampling_fp16" if p.storage == _abi.STORAGE_FP16 else "resampling"
    if key in PROFILED_TRAFFIC:
        tb, tpx = PROFILED_TRAFFIC[key]
        traffic = tb * (W * H) / tpx
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic,
                "traffic_frac": traffic / (passes["resample_ms"] / 1000.0) / 1e9 / peak if traffic else None,
                "kernel": "resampling kernels (reuse-pass combine / select)",
                "peak_kind": f"{peak_kind} copy bandwidth", "algorithmic_bytes_per_launch": res_bytes,
                "algorithmic_bytes_per_pixel": {k: v / (W * H) for k, v in tally.items()},
                "algorithmic_bytes": "counted on the device for the frame's actual work (statistics level 2)",
                "ms": passes["resample_ms"]}
    n_rays = rays["closest_rays"] + rays["shadow_rays"]
    traversal = {"closest_rays_per_frame": rays["closest_rays"], "shadow_rays_per_frame": rays["shadow_rays"],
                 "shift_closest_rays_per_frame": rays["shift_closest_rays"],
                 "shift_shadow_rays_per_frame": rays["shift_shadow_rays"],
                 "shift_jobs_per_frame": rays["shift_jobs"],
                 "node_visits_per_ray": rays["node_visits"] / max(n_rays, 1),
                 "tri_tests_per_ray": rays["tri_tests"] / max(n_rays, 1),
                 "trace_ms": passes["trace_ms"],
                 "rays_per_s": n_rays / (passes["trace_ms"] / 1000.0) if passes["trace_ms"] > 0 else None,
                 "bvh": sc.bvh_info(),
                 "note": "closest / shadow queue traversal kernels of the path and shift machines; rays of shift "
                         "jobs left for the last shift round are traced inside the step kernel"}
    phases = {k: passes[k] for k in ("trace_ms", "shade_ms", "shift_ms", "resample_ms", "search_ms", "other_ms")}
    pass_ms = {k[:-3]: passes[k] for k in keys[:6]}
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    qual = None
    if args.relmse > 0:
        # relMSE of orbit frame 30 against an FP64-accumulated path-traced
        # reference of that frame's camera
        from crisoptix_b200 import quality

        cam_of = lambda f: scenes.orbit_camera(cam, f, 60)  # noqa: E731
        ref = quality.reference_image(sc, W, H, cam_of(30), p, args.relmse)
        qual = {"reference_spp": args.relmse, "frame": 30}
        for name, storage, motion in (("fp32", _abi.STORAGE_FP32, _abi.MOTION_NONE),
                                      ("fp16", _abi.STORAGE_FP16, _abi.MOTION_NONE),
                                      ("fp32_reproject", _abi.STORAGE_FP32, _abi.MOTION_REPROJECT)):
            q = copy.copy(p)
            q.storage = storage
            q.motion_mode = motion
            qual[name] = quality.score(sc, W, H, cam_of, q, 31, args.relmse, ref=ref)
    cb = None
    if not args.no_cpu_baseline and world == 1:
        cb = cpu_baseline(desc, cam, args.workload, os.cpu_count() or 1, 3, warm=1, scale=args.cpu_scale)
        cb.pop("ms_per_frame", None)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_frame, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_for(args.workload, W, H, sc.num_triangles, p, ppp, world, not args.no_graph),
            "launch": tuned if tuned is not None else {"trace_block": 128, "trace_grid": 8,
                                                       "jobs_per_pixel": r.job_capacity()},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 48, "d2h_bytes_per_step": W * H * 12,
                    "copies": "each frame's RGB copied to pinned host memory on a copy stream, overlapping the "
                              "next frame (two output buffers)"},
            "roofline": roofline, "traversal": traversal, "phases_ms": phases, "pass_ms": pass_ms,
            "cpu_baseline": cb, "clocks": clk,
            "gpu_launches": launches_per_frame * args.steps, "image_mean": img_mean, "tonemap": tone,
            "memory": {"renderer_bytes": renderer_bytes, "bytes_per_pixel": renderer_bytes / (W * H),
                       "note": "device memory the renderer allocates (free memory before and after creating it)"}}
    if qual is not None:
        line["quality"] = qual
    if arms is not None:
        line["arms"] = arms
    print(json.dumps(line), flush=True)


def adjoint_time(sc, cam, W: int, H: int, p, warmup: int, steps: int) -> dict:
    """Device time of the resampled estimator's adjoint (crisb_restir_adjoint_*)
    on the workload's last frame: the backward pass for dLoss/dimage = 1 and
    the frozen estimator's evaluation, each averaged over `steps` calls after
    a frame of the orbit, beside that frame's time."""
    import torch

    from crisoptix_b200 import Renderer, scenes

    r = Renderer(W, H, sc, p)
    r.restir_adjoint_enable(True)
    out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    ones = torch.ones(W * H * 3, dtype=torch.float32, device="cuda")
    g_mat = torch.zeros(len(sc.desc.materials) * 7, dtype=torch.float32, device="cuda")
    g_em = torch.zeros(len(sc.desc.emitters) * 3, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    with torch.cuda.stream(stream):
        for f in range(warmup):
            r.launch_frame(scenes.orbit_camera(cam, f, 60), out.data_ptr(), sptr)
        ev[0].record(stream)
        r.launch_frame(scenes.orbit_camera(cam, warmup, 60), out.data_ptr(), sptr)
        ev[1].record(stream)
        r.restir_adjoint_backward(ones.data_ptr(), g_mat.data_ptr(), g_em.data_ptr(), sptr)  # warm-up call
        ev[2].record(stream)
        for _ in range(steps):
            r.restir_adjoint_backward(ones.data_ptr(), g_mat.data_ptr(), g_em.data_ptr(), sptr)
        ev[3].record(stream)
        ev[4].record(stream)
        for _ in range(steps):
            r.restir_adjoint_forward(out.data_ptr(), sptr)
        ev[5].record(stream)
    torch.cuda.synchronize()
    r.check_device_errors()
    frame_ms = ev[0].elapsed_time(ev[1])
    back_ms = ev[2].elapsed_time(ev[3]) / steps
    fwd_ms = ev[4].elapsed_time(ev[5]) / steps
    nonzero = int((g_mat != 0).sum()) + int((g_em != 0).sum())
    del r
    return {"ms_backward": back_ms, "ms_forward": fwd_ms, "ms_frame": frame_ms,
            "backward_over_frame": back_ms / frame_ms, "gradient_entries_nonzero": nonzero,
            "note": "crisb_restir_adjoint_backward with dLoss/dimage = 1 (7 floats per material, 3 per emitter) "
                    "and crisb_restir_adjoint_forward on the last frame of the orbit, FP32 storage"}


def multiview_time(storage: int, batched: bool, steps: int, warmup: int, motion: int = 0) -> dict:
    """Device-resident frames of the 16-view workload (seed 2): ms per frame
    and resampled paths/s.  Renderers are freed on return."""
    import torch

    from crisoptix_b200 import Batch, Renderer, Scene, scenes

    desc, _, _, _, ppp = workload("large")
    sc = Scene(desc)
    p = params_for("large", sc.scene_size)
    p.seed = 2
    p.storage = storage
    p.motion_mode = motion
    views = scenes.multiview_cameras(seed=2)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rs = [Renderer(w, h, sc, p) for _, w, h in views]
    torch.cuda.synchronize()
    mem = free0 - torch.cuda.mem_get_info()[0]
    outs = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for _, w, h in views]
    ptrs = [o.data_ptr() for o in outs]
    px = sum(w * h for _, w, h in views)
    stream = torch.cuda.Stream()
    batch = Batch(rs) if batched else None

    def frame(f):
        cs = [scenes.orbit_camera(c, f % 30, 60) for c, _, _ in views]
        if batch is not None:
            batch.render(cs, ptrs, stream.cuda_stream)
        else:
            for r, c, o in zip(rs, cs, ptrs):
                r.launch_frame(c, o, stream.cuda_stream)

    with torch.cuda.stream(stream):
        for f in range(warmup):
            frame(f)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for f in range(steps):
        frame(warmup + f)
    t1.record(stream)
    torch.cuda.synchronize()
    for r in rs:
        r.check_device_errors()
    ms = t0.elapsed_time(t1) / steps
    del batch, rs, outs
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return {"ms_per_frame": ms, "value": ppp * px * 1000.0 / ms, "pixels": px, "renderer_bytes": mem}


def run_multiview(args):
    """16 views of uneven resolution (8 x 512^2, 4 x 1280x720, 4 x 1920x1080)
    of the large scene, 30-frame sequences; batched = one CUDA graph with a
    branch per view each frame, plain (--no-batch) = the views one after
    another on one stream.  One GPU (views shard across GPUs as replicas)."""
    import torch

    from crisoptix_b200 import Batch, Renderer, Scene, _abi, scenes

    torch.cuda.set_device(0)
    desc, cam0, _, _, ppp = workload("large")
    sc = Scene(desc)
    p = params_for("large", sc.scene_size)
    p.seed = 2
    p.storage = _abi.STORAGE_FP16 if args.storage == "fp16" else _abi.STORAGE_FP32
    p.motion_mode = _abi.MOTION_REPROJECT if args.motion == "reproject" else _abi.MOTION_NONE
    views = scenes.multiview_cameras(seed=2)
    rs = [Renderer(w, h, sc, p) for _, w, h in views]
    outs = [torch.zeros(w * h * 3, dtype=torch.float32, device="cuda") for _, w, h in views]
    ptrs = [o.data_ptr() for o in outs]
    px = sum(w * h for _, w, h in views)
    stream = torch.cuda.Stream()
    batch = None if args.no_batch else Batch(rs)

    def cams(f):  # each view orbits about the room's vertical axis, 30 frames per sequence
        return [scenes.orbit_camera(c, f % 30, 60) for c, _, _ in views]

    def frame(f):
        cs = cams(f)
        if batch is not None:
            batch.render(cs, ptrs, stream.cuda_stream)
        else:
            for r, c, o in zip(rs, cs, ptrs):
                r.launch_frame(c, o, stream.cuda_stream)

    with torch.cuda.stream(stream):
        for f in range(args.warmup):
            frame(f)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for f in range(args.steps):
        frame(args.warmup + f)
    t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    for r in rs:
        r.check_device_errors()
    value = ppp * px * args.steps / (ms / 1000.0)
    launches = sum(r.stats()["kernel_launches"] for r in rs)
    # end to end: every view's image into pinned host memory each frame, on a
    # copy stream that overlaps the next frame (two sets of output buffers;
    # a frame waits for the copies that last read its set)
    out_sets = [outs, [torch.zeros_like(o) for o in outs]]
    host_sets = [[torch.empty(o.numel(), dtype=torch.float32, pin_memory=True) for o in outs] for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [None, None]

    def frame_into(f, j):
        cs = cams(f)
        ps = [o.data_ptr() for o in out_sets[j]]
        if batch is not None:
            batch.render(cs, ps, stream.cuda_stream)
        else:
            for r, c, o in zip(rs, cs, ps):
                r.launch_frame(c, o, stream.cuda_stream)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for f in range(args.steps):
        j = f % 2
        if copied[j] is not None:
            stream.wait_event(copied[j])
        frame_into(args.warmup + f, j)
        rendered = torch.cuda.Event()
        rendered.record(stream)
        copy_stream.wait_event(rendered)
        with torch.cuda.stream(copy_stream):
            for h, o in zip(host_sets[j], out_sets[j]):
                h.copy_(o, non_blocking=True)
        copied[j] = torch.cuda.Event()
        copied[j].record(copy_stream)
    stream.wait_stream(copy_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = e0.elapsed_time(e1)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"multiview: 16 views (8x512x512, 4x1280x720, 4x1920x1080) of the large scene, "
                                   f"{sc.num_triangles} triangles, {px} pixels, "
                                   f"{'FP16' if p.storage == _abi.STORAGE_FP16 else 'FP32'} storage",
                       "batched": batch is not None, "paths_per_pixel": ppp,
                       "l2": "working set larger than L2"},
            "e2e": {"value": ppp * px * args.steps / (e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": 48 * 16,
                    "d2h_bytes_per_step": px * 12,
                    "copies": "every view's RGB copied to pinned host memory on a copy stream, overlapping the "
                              "next frame (two sets of output buffers)"},
            "clocks": clk, "gpu_launches": launches * args.steps,
            "image_mean": float(sum(float(o.mean()) for o in outs) / len(outs))}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="crisb", choices=["crisb", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "small", "multiview"])
    ap.add_argument("--no-batch", action="store_true", help="multiview: render the views one after another")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--relmse", type=int, default=0, metavar="SPP",
                    help="also score orbit frame 30, with FP32 and with FP16 storage, by relMSE against one "
                         "SPP-sample FP64-accumulated path-traced reference")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16"],
                    help="reservoir storage between passes and frames (fp16: packed binary16 / octahedral records)")
    ap.add_argument("--motion", default="none", choices=["none", "reproject"],
                    help="temporal reprojection of the previous reservoirs (off in the reference)")
    ap.add_argument("--autotune", action="store_true", help="pick the traversal launch shape by timing candidates")
    ap.add_argument("--no-graph", action="store_true", help="launch kernels directly instead of one CUDA graph per frame")
    ap.add_argument("--cpu-scale", type=int, default=2)
    ap.add_argument("--res", default=None, help="WxH override of the workload resolution (profiling runs)")
    ap.add_argument("--no-arms", action="store_true",
                    help="skip the comparison arms (FP16 storage, multiview plain vs batched, relMSE)")
    ap.add_argument("--arm-steps", type=int, default=0,
                    help="timed frames of the FP16 single-view arm (0: the main loop's --steps, same frames)")
    ap.add_argument("--arm-mv-steps", type=int, default=4, help="timed frames of each multiview arm")
    ap.add_argument("--arm-ref-spp", type=int, default=256,
                    help="samples per pixel of the path-traced relMSE reference of the arms")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "multiview":
        run_multiview(args)
    else:
        run_crisb(args)


if __name__ == "__main__":
    main()
