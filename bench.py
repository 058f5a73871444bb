#!/usr/bin/env python
"""Benchmark of the NEE path-tracing hot path (RenderingMethod::PATHTRACER).

Default workload (--scene heightfield): the seeded 1M-triangle scene (fBm
heightfield cropped to 1,000,000 triangles in 32x32-quad MESH chunks + 200
subdivision-4 icospheres = 2,024,000 triangles, Lambert / GGX / dielectric
materials, 2048x1024 procedural sky), 1920x1080, max trace depth 8, Russian
roulette off.  --scene cornell: the Cornell box the reference renders
(512x512, depth 5).  A step is one sample per pixel (one PBRenderer::render,
PathTracer.cu:97-169); the timed region renders K steps through
render_frames, which folds several frames into one wavefront.

Metric: Mpaths/s (paths = pixel samples).  `value` is device time of the K
frames with the scene resident in HBM; `e2e` times K single-frame steps
through the public API, each with the tone-mapped RGBA8 frame read back to
pinned host memory.  The 1M-triangle inputs (222 MB resident) exceed the
126 MB L2; the Cornell box does not (stated in config.l2).
`reference_cuda` is the reference's own CUDA path (oracle/_ref/libref_cuda.so,
built for sm_100a with -use_fast_math) timed live on the same GPU.

--scene cache: the radiance cache on the same 1M-triangle scene.  `value` is
plain MSE / cached MSE against a 1024-spp ground truth when the cached
renderer (online training included) gets the device time of `steps` plain
frames (default 16); rows for 4 and 64 frames of budget are added.  The
roofline is the tensor-core inference kernel's against the dense f16/bf16
peak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--scene cornell|medium|batch|cache]
(default K = 256 steps: the configuration's full 256 samples per pixel)
N > 1 runs one process per GPU under torchrun: every rank renders its own
disjoint sample frames (weak scaling, no collective in the timed region).
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCH_PATHS = 1 << 25  # paths per wavefront of the path tracer lines
CACHE_BATCH_PATHS = 1 << 25  # the radiance cache's default wavefront (cupbr_cache_set_batch_paths)

SCENES = {
    "heightfield": dict(
        W=1920, H=1080, DEPTH=8,
        metric="Mpaths/s (NEE path tracing, 1 spp per step, 1M-triangle scene)",
        workload="1M-triangle heightfield + 200 icospheres (2,024,000 tris), 1920x1080, depth 8, "
                 "Lambert/GGX/dielectric, 2048x1024 sky, 1 spp per step",
        l2="inputs larger than L2 (scene 222 MB resident)", ref_res=(960, 540), ref_frames=1),
    "medium": dict(
        W=512, H=512, DEPTH=5, GRID=256, MAJORANT=8.0, MAJORANT_W=8.5, ALBEDO=0.9, G=0.3, FD_SPP=8,
        metric="Mpaths/s (density-grid medium, delta tracking, 1 spp per step)",
        workload="Cornell box filled with a 256^3 4-octave Perlin density grid (seed 0, max sigma_t 8, majorant 8), "
                 "HG g 0.3, albedo 0.9, 512x512, depth 5, analog delta tracking + ratio-tracked light terms, "
                 "1 spp per step",
        l2="density grid 64 MB fits in L2; queues 4M paths 700 MB"),
    "batch": dict(
        W=0, H=0, DEPTH=5,
        metric="Mpaths/s (batched multi-view path tracing: 64 views over 8 scenes per step)",
        workload="8 scenes (4 seeded Cornell variants, 4 seeded 2,024,000-triangle heightfields, each with a "
                 "1024x1024 RGB FP32 albedo texture U[0.2, 0.8]) x 8 views, resolutions from {128^2, 256^2, 512^2, "
                 "1024x768}, spp from {16, 64, 256} (seed 3), depth 5, one persistent-kernel launch in a captured "
                 "CUDA graph per step (autotuned), texture adjoint by path replay",
        l2="heightfield scenes 230 MB each, larger than L2"),
    "cache": dict(
        W=1920, H=1080, DEPTH=8, GT_SPP=1024, CACHE_DEPTH=0, TRAIN_STRIDE=32, LR=1e-2, CACHE_WARMUP=128,
        E2E_FRAMES=2,
        metric="equal-time MSE reduction of the radiance-cached path tracer vs plain NEE path tracing "
               "(plain MSE / cached MSE, 1M-triangle scene)",
        workload="1M-triangle heightfield + 200 icospheres (2,024,000 tris), 1920x1080, depth 8, "
                 "radiance cache (96-64x5-3 FP16 MLP, 12-band position encoding) answering primary hits, "
                 "1 training path per 32, 2^16 samples per frame in Adam steps of 2^14, lr 1e-2; "
                 "time budget = `steps` frames of the plain path tracer",
        l2="inputs larger than L2 (scene 222 MB resident)"),
    "rmse": dict(
        W=1920, H=1080, DEPTH=8, GT_SPP=8192, PIXELS=16, SPP=(1, 4, 16, 64, 256),
        metric="Mpaths/s at equal RMSE vs an FP64 oracle (NEE path tracing, 1M-triangle scene)",
        workload="1M-triangle heightfield + 200 icospheres (2,024,000 tris), 1920x1080, depth 8; RMSE of 16 seeded "
                 "pixels against an 8192-spp FP64 oracle render of them (disjoint sample frames), at 1..256 spp, "
                 "for this library and for the reference's host build",
        l2="inputs larger than L2 (scene 222 MB resident)"),
    "volume": dict(
        W=512, H=512, DEPTH=5,
        metric="Mpaths/s (RenderingMethod::VOLUME, 1 spp per step)",
        workload="VOLUME method: Cornell box with a thin scene medium, a VOLUME sphere behind a glass interface, "
                 "a VOLUME cube, a mirror and a glass sphere, point + area light; 512x512, depth 5, 1 spp per step",
        l2="scene fits in L2; image 3 MB"),
    "gdpt": dict(
        W=512, H=512, DEPTH=5,
        metric="Mpixel-samples/s (RenderingMethod::GRADIENTDOMAIN: base + 4 shift paths and the 50-pass "
               "reconstruction per pixel and step)",
        workload="GRADIENTDOMAIN method on the Cornell box, 512x512, depth 5, 1 sample (5 paths) per pixel per step, "
                 "50 reconstruction passes per step",
        l2="scene and the nine 3 MB images fit in L2"),
    "post": dict(
        W=7680, H=4320, DEPTH=0,
        metric="Mpixels/s (bloom (levels 0-1, PostProcessor::bloom semantics) + Reinhard tone map to RGBA8)",
        workload="bloom with the threshold curve (1, 1) and Reinhard tone map (exposure 1) of a seeded HDR image, "
                 "7680x4320",
        l2="HDR image 398 MB, larger than L2"),
    "cornell": dict(
        W=512, H=512, DEPTH=5,
        metric="Mpaths/s (NEE path tracing, 1 spp per step, Cornell box)",
        workload="Cornell box: 5 quads + two rotated 12-triangle boxes, 0.25x0.25 area light, 512x512, depth 5, "
                 "Lambertian, 1 spp per step",
        l2="scene fits in L2 (a few KB); image and queues 30 MB", ref_res=(512, 512), ref_frames=64),
}


def scenes_module(standalone: bool = False):
    """The seeded scene generators (cupbr_b200/scenes.py).  standalone=True
    loads that file on its own, without the package and so without its native
    library: the reference arm describes the same scene as plain arrays and
    maps no code of this library."""
    if not standalone:
        from cupbr_b200 import scenes
        return scenes
    import importlib.util
    mod = sys.modules.get("_cupbr_scenes_plain")
    if mod is None:
        spec = importlib.util.spec_from_file_location("_cupbr_scenes_plain",
                                                      os.path.join(ROOT, "cupbr_b200", "scenes.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["_cupbr_scenes_plain"] = mod
        spec.loader.exec_module(mod)
    return mod


def make_scene(name, standalone: bool = False):
    scenes = scenes_module(standalone)
    if name in ("heightfield", "cache"):
        return scenes.heightfield_spheres(seed=0)
    return scenes.medium_scene() if name == "medium" else scenes.cornell_box()


def path_config(cfg, args, world: int, desc) -> dict:
    """The `config` dict of the path-tracer lines (heightfield, cornell), the
    same in both arms: a function of the workload and the command line only."""
    W, H = cfg["W"], cfg["H"]
    per_wave = max(1, min(args.steps, BATCH_PATHS // (W * H)))
    return {"workload": cfg["workload"], "width": W, "height": H, "max_trace_depth": cfg["DEPTH"],
            "spp_per_step": 1, "russian_roulette": False, "l2": cfg["l2"], "data": "synthetic, seed 0",
            "parallelism": f"replicas{world}", "triangles": desc.triangle_count(),
            "frames_per_wavefront": per_wave, "wavefront_paths": BATCH_PATHS,
            "warmup_frames": max(args.warmup, per_wave)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---- replicas: one process per GPU, each rendering its own sample frames ----
def init_replicas(backend: str = "nccl"):
    """Process group for N > 1 (rendezvous from the torchrun environment);
    returns (world, rank, local rank)."""
    world, rank, local = _dist()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def frame_base(rank: int) -> int:
    """First sample frame of a rank: ranks render disjoint frames of the same
    view (weak scaling; no collective touches the images)."""
    return rank * 1000000


def max_over_ranks(values, device="cuda"):
    """Each timing as the maximum over ranks (the job is as slow as its
    slowest replica); identity for one process."""
    import torch
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t]


def finish_replicas() -> None:
    import torch
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def settle(self, seconds: float = 0.5) -> None:
        """Waits until nvidia-smi has written its first sample (its start-up
        takes driver locks), at most `seconds`."""
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < seconds:
            try:
                if os.path.getsize(self.path) > 0:
                    return
            except OSError:
                pass
            time.sleep(0.02)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_sample(desc, cfg, seconds: float, threads: int):
    """The reference's own path (oracle/_ref host build) on a bounded pixel
    sample of the same workload; returns (Mpaths/s, kind, sample description)."""
    import numpy as np
    from oracle.bridge import CheckerScene, ref_lib
    W, H, DEPTH = cfg["W"], cfg["H"], cfg["DEPTH"]
    kind = "reference" if ref_lib() is not None else "port"
    sc = CheckerScene(desc, "ref" if kind == "reference" else "oracle")
    cam = np.array([0, 0, 0, np.float32(W) / np.float32(H), 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
    rng = np.random.default_rng(0)
    n = 64
    total_paths, total_t = 0, 0.0
    while total_t < seconds:
        px = np.sort(rng.choice(W * H, min(n, W * H), replace=False)).astype(np.uint32)
        t0 = time.perf_counter()
        sc.pathtrace(cam, W, H, 0, 1, DEPTH, pixels=px, threads=threads)
        dt = time.perf_counter() - t0
        total_paths += len(px)
        total_t += dt
        n = int(min(max(n * 2, 64), max(64, n * (seconds - total_t) / max(dt, 1e-3))))
    what = ("reference object BVH + reference geometry/BSDF code compiled for the host" if kind == "reference"
            else "oracle restatement")
    sample = (f"{total_paths} random pixels of the {W}x{H} frame, 1 spp each, depth {DEPTH}, {what}, "
              f"{threads} threads, {total_t:.1f} s")
    return total_paths / total_t / 1e6, kind, sample


def reference_cuda(desc, cfg):
    """The reference's CUDA path on this GPU (same scene, same camera frustum)."""
    from oracle import bridge
    if bridge.ref_cuda_lib() is None:
        return None
    import cupbr_b200 as cb
    w, h = cfg["ref_res"]
    frames = cfg["ref_frames"]
    rs = bridge.RefCudaScene(desc)
    cam = cb.Camera(w, h).flat()
    rs.pathtrace(cam, w, h, 0, 1, cfg["DEPTH"])  # warm-up
    _, ms = rs.pathtrace(cam, w, h, 0, frames, cfg["DEPTH"])
    return {"value": w * h * frames / (ms * 1e-3) / 1e6, "unit": "Mpaths/s", "ms": ms,
            "resolution": f"{w}x{h}", "frames": frames,
            "kind": "reference PBRendering::pathtracing, sm_100a, -use_fast_math, same GPU"}


def equal_rmse(desc, cfg, threads: int):
    """RMSE against a converged FP64 oracle image (64x64, 4096 spp on the
    host, sample frames disjoint from the compared ones) of this library and
    of the reference's CUDA build at the same spp: equal RMSE at equal spp
    makes the Mpaths/s ratio the equal-RMSE ratio."""
    import numpy as np
    import cupbr_b200 as cb
    from oracle import bridge
    from oracle.bridge import CheckerScene
    w = h = 64
    depth = cfg["DEPTH"]
    cam = cb.Camera(w, h)
    t0 = time.perf_counter()
    f0, n = 1 << 20, 4096
    conv, _ = CheckerScene(desc, "oracle").pathtrace(cam.flat(), w, h, f0, n, depth, threads=threads, precision=64)
    conv = conv * ((f0 + n) / n)  # a running mean started from zero at frame f0 holds sum / (f0 + n)
    t_conv = time.perf_counter() - t0
    sc = desc.build()
    ref = bridge.RefCudaScene(desc) if bridge.ref_cuda_lib() is not None else None
    rows = []
    for spp in (4, 16, 64, 256):
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(depth)
        r.set_russian_roulette(False)
        r.render_frames(cam, spp)
        ours = r.get_output_image().numpy().reshape(-1, 3).astype(np.float64)
        row = {"spp": spp, "rmse": float(np.sqrt(np.mean((ours - conv) ** 2)))}
        if ref is not None:
            theirs, _ = ref.pathtrace(cam.flat(), w, h, 0, spp, depth)
            row["reference_cuda_rmse"] = float(np.sqrt(np.mean((theirs.astype(np.float64) - conv) ** 2)))
        rows.append(row)
    return {"image": f"{w}x{h}", "ground_truth": f"oracle FP64, 4096 spp ({t_conv:.1f} s on {threads} threads)",
            "curve": rows}


def run_reference(args) -> int:
    world, rank, _ = _dist()
    if rank != 0:
        return 0
    cfg = SCENES[args.scene]
    desc = make_scene(args.scene, standalone=True)
    threads = os.cpu_count() or 1
    per_step = max(0.2, args.reference_seconds / max(1, args.steps))
    for _ in range(args.warmup):
        cpu_reference_sample(desc, cfg, 0.2, threads)
    vals = []
    t0 = time.perf_counter()
    kind = sample = None
    for _ in range(args.steps):
        v, kind, sample = cpu_reference_sample(desc, cfg, per_step, threads)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = sum(vals) / len(vals)
    config = path_config(cfg, args, world, desc)
    line = {"metric": cfg["metric"], "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) recorded from
# ncu captures of the dominant kernels: a profiler figure, not measured in the
# bench run (the bench never runs under ncu).  Each entry names the capture;
# the per-kernel summary under profiles/ gives the full command.
NCU_TRAFFIC = {
    # k_extend, heightfield at 960x540 (the bench's scene, smaller frame):
    # 68.5 B per ray on the depth-0 launch, scaled to the 7,769,878 rays of a
    # 1920x1080 two-frame launch (traffic grows with the rays traced)
    "k_extend heightfield": {"bytes_per_launch": 532.2e6,
                             "capture": "ncu --set full -k regex:k_extend -s 8 -c 2, bench.py --resolution 960x540"},
    # k_rc_infer with component-major query records, one cached 4-frame
    # 960x540 wavefront (about 1.54 M queries): read 97.7 + write 9.3 B per
    # query (traffic per query does not depend on the frame size)
    "k_rc_infer heightfield": {"bytes_per_query": 107.0,
                               "capture": "ncu --set full -k regex:k_rc_infer -s 4 -c 1, bench.py --scene cache "
                                          "--resolution 960x540 --batch-paths 4194304 --cache-batch-paths 4194304"},
}


def _read_traffic(scene):
    """Recorded DRAM bytes per k_extend launch for `scene` (NCU_TRAFFIC), or None."""
    rec = NCU_TRAFFIC.get(f"k_extend {scene}")
    return None if rec is None else rec["bytes_per_launch"]


def run_b200(args) -> int:
    import torch
    import cupbr_b200 as cb

    cfg = SCENES[args.scene]
    W, H, DEPTH = cfg["W"], cfg["H"], cfg["DEPTH"]
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)

    desc = make_scene(args.scene)
    sc = desc.build()
    info = sc.info()
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(W, H)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(DEPTH)
    r.set_russian_roulette(False)
    # 32M-path wavefronts (16 frames of 1080p): fewer launches and queue
    # drains per frame; 168 B per path and workspace (5.6 GB each, three with
    # the two pipelined ones)
    r.set_batch_paths(BATCH_PATHS)
    stream = torch.cuda.Stream()
    r.set_stream(stream)
    cam = cb.Camera(W, H)
    r.set_frame_index(frame_base(rank))

    # one instrumented (untimed) frame: ray and traversal counts
    r.set_instrumented(True)
    r.render(cam)
    st = r.stats()
    r.set_instrumented(False)
    sampler = ClockSampler(local)  # started before the warm-up: its start-up must not fall in the timed region
    # warm-up: at least W frames and one full wavefront, so the wavefront
    # workspaces are allocated before any timed pass
    per_wave = max(1, min(args.steps, BATCH_PATHS // (W * H)))
    warm = max(args.warmup, per_wave)
    r.render_frames(cam, warm)
    torch.cuda.synchronize()
    sampler.settle()
    if world > 1:
        torch.distributed.barrier()

    # stage times: the same K frames on one stream with CUDA events between
    # the stages (the roofline's kernel times; overlapped wavefronts cannot
    # be timed stage by stage)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r.set_profiling(True)
    torch.cuda.synchronize()
    e0.record(stream)
    r.render_frames(cam, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    r.set_profiling(False)
    stages = r.stage_times()
    ms_one_stream = e0.elapsed_time(e1)

    # the timed region: render_frames with the wavefronts alternating between
    # the renderer's two internal streams (set_pipelined), folded into the
    # image on `stream` in frame order
    r.set_pipelined(True)
    r.render_frames(cam, warm)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    r.render_frames(cam, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms = e0.elapsed_time(e1)
    repeats_ms = [ms]
    if args.repeats > 1:
        # further timed regions of the same K frames; the value is their median
        for _ in range(args.repeats - 1):
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            r.render_frames(cam, args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
            repeats_ms.append(e0.elapsed_time(e1))
        ms = _median(repeats_ms)
    clocks = sampler.stop()
    errors = r.error_count()

    # end to end through the public API: render + tone map + RGBA8 readback per
    # step, render() pipelined (the next frame traces while this one is tone
    # mapped and read back)
    r.set_pipelined(True)
    tm = cb.ToneMapper(cb.ToneMappingType.REINHARD)
    tm.set_stream(stream)
    tm.register_image(r.get_output_image())
    rgba = tm.get_render_buffer()
    host = torch.empty(rgba.nbytes, dtype=torch.uint8, pin_memory=True)
    for _ in range(4):  # every internal stream's workspace allocated before the timed region
        r.render(cam)
        tm.tone_map()
        cb._native.call("cupbr_memcpy_d2h", host.data_ptr(), rgba.ptr, rgba.nbytes, stream.cuda_stream)
    torch.cuda.synchronize()
    cam_bytes = cb._native.C.sizeof(cb._native.Camera)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        r.render(cam)  # the camera pose is read from host memory by this call
        tm.tone_map()
        cb._native.call("cupbr_memcpy_d2h", host.data_ptr(), rgba.ptr, rgba.nbytes, stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)

    ms, ms_e2e, ms_one_stream = max_over_ranks([ms, ms_e2e, ms_one_stream])

    paths = W * H * args.steps * world
    value = paths / (ms * 1e-3) / 1e6
    e2e = paths / (ms_e2e * 1e-3) / 1e6
    rays_per_frame = st["ext_rays"] + st["shadow_rays"]

    # roofline of the dominant kernel (k_extend, closest hit)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    ext_bytes_frame = 112.0 * st["ext_nodes"] + 48.0 * st["ext_prims"] + 96.0 * st["ext_rays"]
    launches = max(1, stages["extend_launches"])
    per_launch = ext_bytes_frame * args.steps / launches
    avg_launch_s = stages["extend"] / launches * 1e-3
    achieved = per_launch / avg_launch_s / 1e9 if avg_launch_s > 0 else 0.0
    traffic = _read_traffic(args.scene)
    # the shadow-ray kernel (k_connect) on the same model: node and triangle
    # reads of its occlusion traversals + 48 B entry read + 16 B radiance update per ray
    con_bytes_frame = 112.0 * st["shadow_nodes"] + 48.0 * st["shadow_prims"] + 64.0 * st["shadow_rays"]
    con_per_launch = con_bytes_frame * args.steps / launches
    con_avg_s = stages["connect"] / launches * 1e-3
    con_achieved = con_per_launch / con_avg_s / 1e9 if con_avg_s > 0 else 0.0

    if rank == 0:
        config = path_config(cfg, args, world, desc)
        assert config["triangles"] == info["triangles"] and config["warmup_frames"] == warm
        line = {"metric": cfg["metric"], "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "e2e": {"value": e2e, "unit": "Mpaths/s", "h2d_bytes_per_step": cam_bytes,
                        "d2h_bytes_per_step": rgba.nbytes,
                        "note": "render + tone map + RGBA8 readback per step; render() pipelined (set_pipelined)"},
                "timed": "render_frames(K) with set_pipelined: the wavefronts alternate between two internal streams "
                         "and workspaces and are folded into the image in frame order on the caller's stream"
                         + (f"; median of {args.repeats} timed regions of K frames" if args.repeats > 1 else ""),
                "repeats_ms": repeats_ms,
                "one_stream": {"value": paths / (ms_one_stream * 1e-3) / 1e6, "unit": "Mpaths/s",
                               "note": "the same K frames on one stream with stage events (stage_ms_per_step, roofline)"},
                "mrays_per_s": rays_per_frame * args.steps * world / (ms * 1e-3) / 1e6,
                "rays_per_frame": {"extension": st["ext_rays"], "shadow": st["shadow_rays"]},
                "traversal_per_ray": {
                    "closest_hit": {"node_visits": st["ext_nodes"] / max(1, st["ext_rays"]),
                                    "primitive_tests": st["ext_prims"] / max(1, st["ext_rays"])},
                    "shadow": {"node_visits": st["shadow_nodes"] / max(1, st["shadow_rays"]),
                               "primitive_tests": st["shadow_prims"] / max(1, st["shadow_rays"])}},
                "stage_ms_per_step": {k: round(stages[k] / args.steps, 4)
                                      for k in ("camera", "extend", "shade", "connect", "accumulate")},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_src} hbm_gbs",
                             "kernel": "k_extend (closest hit), timed as the closest-hit stage of the one-stream pass, "
                                       "which also holds the camera-ray packets and the per-path tail kernel",
                             "bytes_per_launch": per_launch,
                             "bytes_model": "112*node_visits (7 float4 of a 4-wide node) + 48*triangle_tests + 96 per ray"},
                "roofline_connect": {"bound": "hbm", "achieved": con_achieved, "peak": peak, "unit": "GB/s",
                                     "frac": con_achieved / peak, "peak_source": f"{peak_src} hbm_gbs",
                                     "kernel": "k_connect (shadow rays, any hit), timed as the shadow-ray stage of the "
                                               "one-stream pass",
                                     "bytes_per_launch": con_per_launch,
                                     "bytes_model": "112*node_visits + 48*triangle_tests + 64 per shadow ray"},
                "gpu_launches": stages["frames"] * (4 * DEPTH + 2),
                "device_errors": errors,
                "scene": {"triangles": info["triangles"], "bvh_nodes": info["bvh_nodes"],
                          "device_mb": round(info["device_bytes"] / 2**20, 1)},
                "clocks": clocks}
        if world == 1 and not args.no_reference_cuda:
            try:
                line["reference_cuda"] = reference_cuda(desc, cfg)
                if line["reference_cuda"]:
                    line["reference_cuda"]["speedup_of_value"] = value / line["reference_cuda"]["value"]
            except Exception as exc:  # reported, never fatal for the bench line
                line["reference_cuda"] = {"unavailable": str(exc)[:200]}
        if world == 1 and args.scene == "cornell":
            # the same K frames through one persistent-kernel launch (set_persistent)
            r.set_pipelined(False)
            r.set_persistent(True)
            r.render_frames(cam, warm)
            pt = []
            for _ in range(args.repeats):
                torch.cuda.synchronize()
                e0.record(stream)
                r.render_frames(cam, args.steps)
                e1.record(stream)
                torch.cuda.synchronize()
                pt.append(e0.elapsed_time(e1))
            r.set_persistent(False)
            line["persistent_render_frames"] = {
                "value": W * H * args.steps / (_median(pt) * 1e-3) / 1e6, "unit": "Mpaths/s", "repeats_ms": pt,
                "note": "render_frames(K) as one persistent-kernel launch (warps over 8x4 tiles through all K "
                        "frames), same image as the wavefronts"}
        if world == 1 and args.scene == "cornell" and not args.no_cpu_baseline:
            try:
                line["equal_rmse"] = equal_rmse(desc, cfg, os.cpu_count() or 1)
            except Exception as exc:  # reported, never fatal for the bench line
                line["equal_rmse"] = {"unavailable": str(exc)[:200]}
        if world == 1 and not args.no_cpu_baseline:
            v, kind, sample = cpu_reference_sample(desc, cfg, args.cpu_seconds, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": v, "unit": "Mpaths/s", "cores": os.cpu_count() or 1, "kind": kind,
                                    "sample": sample}
        print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def medium_cpu_sample(desc, cfg, grid, seconds: float, threads: int):
    """The oracle's restatement of the grid medium (no reference counterpart)
    on a bounded pixel sample; returns (Mpaths/s, sample description)."""
    import numpy as np
    import cupbr_b200 as cb
    from oracle.bridge import CheckerScene
    W, H, DEPTH = cfg["W"], cfg["H"], cfg["DEPTH"]
    sc = CheckerScene(desc, "oracle")
    cam = cb.Camera(W, H).flat()
    box = (-1, -1, 1, 1, 1, 3)
    rng = np.random.default_rng(0)
    n, total_paths, total_t = 256, 0, 0.0
    while total_t < seconds:
        px = np.sort(rng.choice(W * H, min(n, W * H), replace=False)).astype(np.uint32)
        t0 = time.perf_counter()
        sc.medium_forward(grid, box, cfg["MAJORANT"], cfg["ALBEDO"], cfg["G"], 0.0, cam, W, H, 1, 0, DEPTH,
                          pixels=px, threads=threads)
        dt = time.perf_counter() - t0
        total_paths += len(px)
        total_t += dt
        n = int(min(max(n * 2, 256), max(256, n * (seconds - total_t) / max(dt, 1e-3))))
    sample = (f"{total_paths} random pixels of the {W}x{H} frame, 1 spp each, depth {DEPTH}, oracle restatement "
              f"(float), {threads} threads, {total_t:.1f} s")
    return total_paths / total_t / 1e6, sample


def run_reference_batch(args) -> int:
    """Reference arm of the batch workload: the reference has no batching and
    its host path would take hours on the heightfield views, so it reports
    unavailable (the CUDA build's per-view loop is timed inside the b200 line)."""
    if _dist()[1] == 0:
        print(json.dumps({"impl": "reference", "unavailable": "the reference renders one view per render() call; "
                          "its CUDA build is timed on the Cornell views inside the b200 line"}), flush=True)
    return 0


def run_medium(args) -> int:
    """The density-grid medium workload: forward (analog delta tracking) as
    the headline, then the path-replay gradient of an L2 image loss
    (weighted tracking, majorant 8.5) with a central-difference check."""
    import numpy as np
    import torch
    import cupbr_b200 as cb
    from cupbr_b200 import medium as M
    from cupbr_b200 import scenes

    cfg = SCENES["medium"]
    W, H, DEPTH = cfg["W"], cfg["H"], cfg["DEPTH"]
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)
    desc = make_scene("medium")
    sc = desc.build()
    grid = scenes.perlin_grid(cfg["GRID"], seed=0, sigma_max=8.0)
    box = ((-1.0, -1.0, 1.0), (1.0, 1.0, 3.0))
    dens = torch.from_numpy(grid).cuda()
    stream = torch.cuda.Stream()
    cam = cb.Camera(W, H)
    img = torch.empty((H, W, 3), device="cuda", dtype=torch.float32)
    fwd = M.Medium(grid.shape, box, cfg["MAJORANT"], cfg["ALBEDO"], cfg["G"], 0.0)
    frame0 = frame_base(rank)

    # one instrumented (untimed) wavefront: density lookups and queue sizes
    fwd.set_instrumented(True)
    fwd.forward(sc, dens.data_ptr(), cam, W, H, 1, frame0, DEPTH, img.data_ptr(), stream.cuda_stream)
    st = fwd.stats()
    fwd.set_instrumented(False)
    sampler = ClockSampler(local)
    fwd.forward(sc, dens.data_ptr(), cam, W, H, args.warmup, frame0, DEPTH, img.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    sampler.settle()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fwd.set_profiling(True)
    torch.cuda.synchronize()
    e0.record(stream)
    fwd.forward(sc, dens.data_ptr(), cam, W, H, args.steps, frame0, DEPTH, img.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd.set_profiling(False)
    stages = fwd.stage_times()
    ms = e0.elapsed_time(e1)
    repeats_ms = []
    if args.repeats > 1:
        # unprofiled timed regions of the same K spp; the value is their median
        for _ in range(args.repeats):
            torch.cuda.synchronize()
            e0.record(stream)
            fwd.forward(sc, dens.data_ptr(), cam, W, H, args.steps, frame0, DEPTH, img.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            repeats_ms.append(e0.elapsed_time(e1))
        ms = _median(repeats_ms)
    clocks = sampler.stop()

    # end to end: one C-ABI call per step (1 spp) and the HDR image read back to pinned host memory
    host = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True)
    for k in range(2):
        fwd.forward(sc, dens.data_ptr(), cam, W, H, 1, frame0 + k, DEPTH, img.data_ptr(), stream.cuda_stream)
        cb._native.call("cupbr_memcpy_d2h", host.data_ptr(), img.data_ptr(), img.numel() * 4, stream.cuda_stream)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for k in range(args.steps):
        fwd.forward(sc, dens.data_ptr(), cam, W, H, 1, frame0 + k, DEPTH, img.data_ptr(), stream.cuda_stream)
        cb._native.call("cupbr_memcpy_d2h", host.data_ptr(), img.data_ptr(), img.numel() * 4, stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)

    # gradient of an L2 loss against a target rendered from the perturbed grid
    bwd = M.Medium(grid.shape, box, cfg["MAJORANT_W"], cfg["ALBEDO"], cfg["G"], 0.5)
    rng = np.random.default_rng(1)
    target_grid = (grid * (1.0 + 0.1 * rng.uniform(-1.0, 1.0, grid.shape))).astype(np.float32)
    target_grid = np.minimum(target_grid, np.float32(cfg["MAJORANT_W"] - 0.01))
    tdens = torch.from_numpy(target_grid).cuda()
    target = torch.empty_like(img)
    spp_g = args.steps
    bwd.forward(sc, tdens.data_ptr(), cam, W, H, spp_g, frame0, DEPTH, target.data_ptr(), stream.cuda_stream)
    bwd.forward(sc, dens.data_ptr(), cam, W, H, spp_g, frame0, DEPTH, img.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    grad_img = (2.0 * (img - target)).contiguous()
    gd = torch.zeros_like(dens)
    npar = M.Medium.param_count(sc)
    gp = torch.zeros(npar, device="cuda", dtype=torch.float32)
    bwd.backward(sc, dens.data_ptr(), cam, W, H, 1, frame0, DEPTH, grad_img.data_ptr(), gd.data_ptr(),
                 gp.data_ptr(), stream.cuda_stream)  # warm-up
    torch.cuda.synchronize()
    gd.zero_()
    gp.zero_()
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    bwd.backward(sc, dens.data_ptr(), cam, W, H, spp_g, frame0, DEPTH, grad_img.data_ptr(), gd.data_ptr(),
                 gp.data_ptr(), stream.cuda_stream)
    e5.record(stream)
    torch.cuda.synchronize()
    ms_grad = e4.elapsed_time(e5)

    # central differences (h = 1e-3) on 64 voxels (seed 2) and the medium albedo, at FD_SPP samples
    fd = None
    if rank == 0 and not args.no_fd_check:
        spp_fd = cfg["FD_SPP"]
        gi_fd = None

        def loss(d, medium):
            medium.forward(sc, d.data_ptr(), cam, W, H, spp_fd, frame0, DEPTH, img.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            return float(((img.double() - target.double()) ** 2).sum())

        loss(dens, bwd)
        gi_fd = (2.0 * (img - target)).contiguous()
        g_fd = torch.zeros_like(dens)
        p_fd = torch.zeros(npar, device="cuda", dtype=torch.float32)
        bwd.backward(sc, dens.data_ptr(), cam, W, H, spp_fd, frame0, DEPTH, gi_fd.data_ptr(), g_fd.data_ptr(),
                     p_fd.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        flat = grid.ravel()
        h = 1e-3
        ok = np.flatnonzero((flat > 2e-2) & (flat < cfg["MAJORANT_W"] - 2e-2))
        vox = np.random.default_rng(2).choice(ok, 64, replace=False)
        adj = g_fd.view(-1)[torch.from_numpy(vox).cuda()].cpu().numpy().astype(np.float64)
        dflat = dens.view(-1)
        scale = max(float(np.abs(adj).max()), 1e-30)
        fd_steps = {}
        for hh in (1e-3, 1e-2):
            fds = []
            for k in vox:
                v0 = float(flat[k])
                a, b = np.float32(v0 + hh), np.float32(v0 - hh)
                dflat[int(k)] = float(a)
                fp = loss(dens, bwd)
                dflat[int(k)] = float(b)
                fm = loss(dens, bwd)
                dflat[int(k)] = v0
                fds.append((fp - fm) / (float(a) - float(b)))
            fds = np.array(fds)
            err = np.abs(adj - fds)
            big = np.abs(fds) >= 0.05 * scale
            fd_steps[str(hh)] = {"max_abs_err_over_max_grad": float(err.max() / scale),
                                 "within_1e-3_rel_or_1e-4_of_max": float(np.mean(err <= 1e-3 * np.abs(fds)
                                                                                  + 1e-4 * scale)),
                                 "max_rel_err_where_fd_over_5pct_of_max": float((err[big] / np.abs(fds[big])).max())
                                 if big.any() else None}
        a_alb, b_alb = np.float32(cfg["ALBEDO"] + h), np.float32(cfg["ALBEDO"] - h)
        m_p = M.Medium(grid.shape, box, cfg["MAJORANT_W"], float(a_alb), cfg["G"], 0.5)
        m_m = M.Medium(grid.shape, box, cfg["MAJORANT_W"], float(b_alb), cfg["G"], 0.5)
        fd_alb = (loss(dens, m_p) - loss(dens, m_m)) / (float(a_alb) - float(b_alb))
        adj_alb = float(p_fd[0])
        fd = {"voxels": 64, "voxel_seed": 2, "spp": spp_fd, "loss": "sum of squared differences to target",
              "note": "central differences of float32 images carry rounding noise ~ eps * |I| / h: the "
                      "absolute error falls ~10x from h = 1e-3 to 1e-2",
              "density": fd_steps,
              "albedo": {"h": h, "adjoint": adj_alb, "finite_difference": fd_alb,
                         "rel_err": abs(adj_alb - fd_alb) / max(abs(fd_alb), 1e-30)}}

    errors = fwd.error_count() + bwd.error_count()
    ms, ms_e2e, ms_grad = max_over_ranks([ms, ms_e2e, ms_grad])
    paths = W * H * args.steps * world
    value = paths / (ms * 1e-3) / 1e6

    # roofline of the dominant kernel: k_medium_shade (free flight + vertex)
    # or k_medium_transmit (ratio tracking), by measured stage time
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    npaths = max(1, st["paths"])
    models = {
        "shade": ("k_medium_flight + k_medium_scatter + k_medium_surface",
                  (4.0 * st["flight_lookups"] + 152.0 * st["vertices"] + 64.0 * st["shadow_rays"]
                   + 48.0 * (st["vertices"] - st["paths"])) / npaths,
                  "4 per free-flight density lookup + 56 per entry read + 48 per vertex written and read again "
                  "+ 64 per shadow ray written + 48 per next ray written"),
        "transmit": ("k_medium_transmit",
                     (4.0 * st["ratio_lookups"] + 80.0 * st["shadow_rays"]) / npaths,
                     "4 per ratio-tracking density lookup + 80 per shadow ray (ray, RNG state, term read, "
                     "term written)")}
    top = max(models, key=lambda k: stages[k])
    kname, per_path, bytes_model = models[top]
    launches = max(1, stages["shade_launches"])  # one shade and one transmit launch per depth and wavefront
    per_launch = per_path * W * H * args.steps / launches
    avg_launch_s = stages[top] / launches * 1e-3
    achieved = per_launch / avg_launch_s / 1e9 if avg_launch_s > 0 else 0.0
    if rank == 0:
        config = {"workload": cfg["workload"], "width": W, "height": H, "max_trace_depth": DEPTH,
                  "grid": f"{cfg['GRID']}^3 float32", "majorant": cfg["MAJORANT"], "tracking": "analog delta",
                  "spp_per_step": 1, "l2": cfg["l2"], "data": "synthetic, seed 0",
                  "parallelism": f"replicas{world}", "frames_per_wavefront": max(1, min(args.steps, (1 << 22) // (W * H))),
                  "timing": (f"median of {args.repeats} timed regions of K spp (stage times from one more, "
                             "profiled)") if args.repeats > 1 else "one timed region of K spp (profiled)"}
        line = {"metric": cfg["metric"], "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "e2e": {"value": paths / (ms_e2e * 1e-3) / 1e6, "unit": "Mpaths/s",
                        "h2d_bytes_per_step": cb._native.C.sizeof(cb._native.Camera),
                        "d2h_bytes_per_step": W * H * 12, "note": "one 1-spp C-ABI call + HDR readback per step"},
                "repeats_ms": repeats_ms,
                "per_path": {k: st[k] / npaths
                             for k in ("flight_lookups", "ratio_lookups", "vertices", "shadow_rays")},
                "stage_ms_per_step": {k: round(stages[k] / args.steps, 4)
                                      for k in ("camera", "extend", "shade", "transmit", "connect", "accumulate")},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "peak_source": f"{peak_src} hbm_gbs",
                             "kernel": kname, "bytes_per_launch": per_launch, "bytes_model": bytes_model,
                             "traffic_note": "null: the 64 MB grid stays in L2 in the timed run, so a cold-cache "
                                             "ncu capture's DRAM bytes do not describe it"},
                "gradient": {"mpaths_per_s": W * H * spp_g * world / (ms_grad * 1e-3) / 1e6,
                             "gradients_per_s": world / (ms_grad * 1e-3), "ms": ms_grad, "spp": spp_g,
                             "tracking": "weighted, q 0.5, majorant 8.5",
                             "outputs": f"{grid.size} voxel + {npar} parameter gradients",
                             "fd_check": fd},
                "gpu_launches": stages["wavefronts"] * (4 * DEPTH + 2),
                "device_errors": errors,
                "clocks": clocks,
                "reference_cuda": {"unavailable": "the reference has no density-grid medium (homogeneous only)"}}
        if world == 1 and not args.no_cpu_baseline:
            v, sample = medium_cpu_sample(desc, cfg, grid, args.cpu_seconds, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": v, "unit": "Mpaths/s", "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": sample}
        print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def run_batch(args) -> int:
    """C3: 64 views over 8 scenes as one batched launch (a captured graph of
    a few large wavefronts) vs the same views rendered one render() per
    frame per view, and vs the reference CUDA build's render() loop on the
    Cornell views."""
    import numpy as np
    import torch
    import cupbr_b200 as cb
    from cupbr_b200 import scenes

    cfg = SCENES["batch"]
    DEPTH = cfg["DEPTH"]
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)
    torch.zeros(1, device="cuda")  # CUDA context up before the scene builds are timed
    t0 = time.perf_counter()
    # per scene a 1024x1024 RGB albedo texture (texels U[0.2, 0.8], seeded
    # by (4, scene)) on its white Cornell quads / Lambert terrain chunks
    descs = [scenes.with_texture(scenes.cornell_variant(s) if s < 4 else scenes.heightfield_spheres(seed=s), 1024,
                                 seed=(4, s)) for s in range(8)]
    t1 = time.perf_counter()
    built = [d.build() for d in descs]  # BVHs built on the GPU (the default builder)
    t_build = time.perf_counter() - t1
    bvh_ms = sum(b.info()["bvh_build_ms"] for b in built)
    commit_ms = sum(b.info()["commit_ms"] for b in built)
    # the same eight scenes with the BVHs built on the host's threads, for comparison
    t2 = time.perf_counter()
    host_built = [d.build(bvh_params={"builder": "host"}) for d in descs]
    t_build_host = time.perf_counter() - t2
    bvh_ms_host = sum(b.info()["bvh_build_ms"] for b in host_built)
    del host_built
    rng = np.random.default_rng(3)
    sizes = [(128, 128), (256, 256), (512, 512), (1024, 768)]
    views, specs, imgs = [], [], []
    for si, sc in enumerate(built):
        for _ in range(8):
            w, h = sizes[rng.integers(4)]
            spp = int(rng.choice([16, 64, 256]))
            base = cb.Camera(w, h)
            if si < 4:
                pos = tuple(rng.uniform(-0.3, 0.3, 3))
            else:
                pos = (rng.uniform(-4, 4), rng.uniform(0.5, 2.0), rng.uniform(-1, 3))
            cam = cb.Camera.from_axes(pos, base.x_axis(), base.y_axis(), base.z_axis())
            img = torch.zeros((h, w, 3), device="cuda")
            imgs.append(img)
            specs.append((si, cam, w, h, spp))
            views.append(dict(scene=sc, camera=cam, width=w, height=h, spp=spp, frame0=frame_base(rank),
                              image=img.data_ptr()))
    stream = torch.cuda.Stream()
    batch = cb.Batch(views, DEPTH)
    tuned_ms = batch.autotune(stream.cuda_stream)
    info = batch.info()
    sampler = ClockSampler(local)
    for _ in range(args.warmup):
        batch.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    sampler.settle()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        batch.launch(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)

    # end to end: every step also reads all 64 HDR images back to pinned host memory
    host = [torch.empty(img.shape, dtype=torch.float32, pin_memory=True) for img in imgs]
    d2h = sum(img.numel() * 4 for img in imgs)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        batch.launch(stream.cuda_stream)
        for hb, img in zip(host, imgs):
            cb._native.call("cupbr_memcpy_d2h", hb.data_ptr(), img.data_ptr(), img.numel() * 4, stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)

    # texture adjoint (cupbr_batch_backward) of an L2 loss against a grey
    # target: one timed replay of every path of the step
    gimgs = [(img - 0.5).contiguous() for img in imgs]
    batch.backward([g.data_ptr() for g in gimgs], stream=stream.cuda_stream)
    torch.cuda.synchronize()
    eb0, eb1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    eb0.record(stream)
    batch.backward([g.data_ptr() for g in gimgs], stream=stream.cuda_stream)
    eb1.record(stream)
    torch.cuda.synchronize()
    ms_bwd = eb0.elapsed_time(eb1)
    tex_grads = sum(1 for b in built if b.albedo_texture_or_none() is not None)

    # one launch in each mode (the tuned shape of the persistent kernel, the
    # tuned wavefront size for both wavefront modes), then back to the tuned
    # configuration
    tuned = batch.mode()
    mode_ms = {}
    for mode in ("persistent", "wavefront", "cooperative"):
        if mode == "persistent":
            pers = tuned["mode"] == "persistent"
            batch.set_mode("persistent", tuned["threads_per_block"] if pers else 128,
                           tuned["blocks_per_sm"] if pers else 0, tuned["camera_packets"] if pers else True)
        else:
            batch.set_mode(mode)
        batch.launch(stream.cuda_stream)
        torch.cuda.synchronize()
        e6, e7 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e6.record(stream)
        batch.launch(stream.cuda_stream)
        e7.record(stream)
        torch.cuda.synchronize()
        mode_ms[mode] = e6.elapsed_time(e7)
    batch.set_mode(tuned["mode"], tuned["threads_per_block"], tuned["blocks_per_sm"], tuned["camera_packets"])

    # the same views one PBRenderer.render() per frame (the reference's usage), once
    seq_paths = 0
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    renderers = []
    for (si, cam, w, h, spp) in specs:
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(built[si])
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(DEPTH)
        r.set_russian_roulette(False)
        r.set_stream(stream)
        renderers.append(r)
    torch.cuda.synchronize()
    t_seq0 = time.perf_counter()
    e4.record(stream)
    for r, (si, cam, w, h, spp) in zip(renderers, specs):
        for _ in range(spp):
            r.render(cam)
        seq_paths += w * h * spp
    e5.record(stream)
    torch.cuda.synchronize()
    wall_seq = time.perf_counter() - t_seq0
    ms_seq = max(e4.elapsed_time(e5), wall_seq * 1e3)
    errors = sum(r.error_count() for r in renderers)

    ms, ms_e2e = max_over_ranks([ms, ms_e2e])
    paths = info["paths"] * args.steps * world
    value = paths / (ms * 1e-3) / 1e6
    line = None
    if rank == 0:
        config = {"workload": cfg["workload"], "views": len(views), "scenes": len(built), "max_trace_depth": DEPTH,
                  "paths_per_step": info["paths"], "autotuned": tuned, "autotune_best_ms": tuned_ms,
                  "wavefronts_per_step": info["wavefronts"], "autotuned_batch_paths": info["batch_paths"],
                  "scene_build_s": round(t_build, 2), "scene_generation_s": round(t1 - t0, 2),
                  "scene_commit_ms": round(commit_ms, 1), "bvh_build_ms": round(bvh_ms, 1),
                  "scene_build_s_host_bvh": round(t_build_host, 2), "bvh_build_ms_host": round(bvh_ms_host, 1),
                  "l2": cfg["l2"], "data": "synthetic, seeds 0-7 (scenes), 3 (views)",
                  "parallelism": f"replicas{world}"}
        line = {"metric": cfg["metric"], "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "e2e": {"value": paths / (ms_e2e * 1e-3) / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": d2h, "note": "graph launch + all 64 HDR images read back per step"},
                "gradient": {"texture_gradients_per_s": world / (ms_bwd * 1e-3), "ms": ms_bwd,
                             "mpaths_per_s": info["paths"] * world / (ms_bwd * 1e-3) / 1e6,
                             "outputs": f"{tex_grads} albedo textures of 1024x1024 RGB",
                             "method": "path replay of every path of the step (cupbr_batch_backward)"},
                "modes": {m: {"value": info["paths"] / (t * 1e-3) / 1e6, "unit": "Mpaths/s", "ms": t,
                              "launches": 1 if m != "wavefront" else None}
                          for m, t in mode_ms.items()},
                "sequential_render_calls": {"value": seq_paths / (ms_seq * 1e-3) / 1e6, "unit": "Mpaths/s",
                                            "ms": ms_seq, "render_calls": sum(s[4] for s in specs),
                                            "note": "same views, one PBRenderer.render() per frame, this library"},
                "roofline": None,
                "roofline_note": "the kernels are the path tracer's (k_extend dominant); one graph launch has no "
                                 "per-kernel events -- see the heightfield line",
                "gpu_launches": info["kernel_launches"] * args.steps,
                "device_errors": errors, "clocks": clocks}
        if world == 1 and not args.no_reference_cuda:
            try:
                from oracle import bridge
                if bridge.ref_cuda_lib() is not None:
                    ref_ms, ref_paths, our_ms = 0.0, 0, 0.0
                    cviews = [(i, s) for i, s in enumerate(specs) if s[0] < 4]
                    ref_scenes = {si: bridge.RefCudaScene(descs[si]) for si in range(4)}
                    for i, (si, cam, w, h, spp) in cviews:
                        ref_scenes[si].pathtrace(cam.flat(), w, h, 0, 1, DEPTH)  # warm-up
                        _, m = ref_scenes[si].pathtrace(cam.flat(), w, h, 0, spp, DEPTH)
                        ref_ms += m
                        ref_paths += w * h * spp
                    sub = cb.Batch([views[i] for i, _ in cviews], DEPTH)
                    sub.autotune(stream.cuda_stream)
                    sub.launch(stream.cuda_stream)
                    e6, e7 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e6.record(stream)
                    sub.launch(stream.cuda_stream)
                    e7.record(stream)
                    torch.cuda.synchronize()
                    our_ms = e6.elapsed_time(e7)
                    line["reference_cuda"] = {
                        "value": ref_paths / (ref_ms * 1e-3) / 1e6, "unit": "Mpaths/s", "ms": ref_ms,
                        "views": len(cviews), "batched_value_same_views": ref_paths / (our_ms * 1e-3) / 1e6,
                        "kind": "reference PBRendering::pathtracing per view and frame, sm_100a, -use_fast_math, "
                                "the 32 Cornell-variant views without their textures (the reference has none; its heightfield "
                                "traversal is ~10,000x slower)"}
            except Exception as exc:
                line["reference_cuda"] = {"unavailable": str(exc)[:200]}
        print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def run_rmse(args) -> int:
    """Equal-RMSE comparison on the 1M-triangle workload: the RMSE-vs-spp
    curve of this library and of the reference's host build against an FP64
    oracle render (reference semantics) of a seeded pixel subset.  The two
    curves coincide (the same sample streams, pixel for pixel), so Mpaths/s
    at equal RMSE is the Mpaths/s of each.  Also checks the GPU ground truth
    the radiance-cache line uses (1024 spp) against the same FP64 render."""
    import numpy as np
    import torch
    import cupbr_b200 as cb
    from oracle.bridge import CheckerScene, ref_lib

    cfg = SCENES["rmse"]
    W, H, D = cfg["W"], cfg["H"], cfg["DEPTH"]
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)
    if rank != 0:
        finish_replicas()
        return 0
    desc = make_scene("heightfield")
    sc = desc.build()
    rng = np.random.default_rng(17)
    px = np.sort(rng.choice(W * H, cfg["PIXELS"], replace=False)).astype(np.uint32)
    cam = cb.Camera(W, H)
    threads = os.cpu_count() or 1
    # FP64 oracle ground truth (frames 2^20 .., disjoint from the compared ones)
    t0 = time.perf_counter()
    f0, n = 1 << 20, cfg["GT_SPP"]
    gt, _ = CheckerScene(desc, "oracle").pathtrace(cam.flat(), W, H, f0, n, D, pixels=px, threads=threads,
                                                   precision=64)
    gt = gt * ((f0 + n) / n)
    t_gt = time.perf_counter() - t0
    rmse = lambda a: float(np.sqrt(np.mean((np.asarray(a, np.float64) - gt) ** 2)))
    # this library: full frames, the subset's pixels read at each spp
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(W, H)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(D)
    r.set_russian_roulette(False)
    ours, done = [], 0
    for spp in cfg["SPP"]:
        r.render_frames(cam, spp - done)
        done = spp
        ours.append(rmse(r.get_output_image().numpy().reshape(-1, 3)[px]))
    # throughput of the same renders
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r.render_frames(cam, 64)
    e1.record()
    torch.cuda.synchronize()
    ours_mpaths = W * H * 64 / (e0.elapsed_time(e1) * 1e-3) / 1e6
    # the reference's host build on the subset, the running mean continued
    kind = "reference" if ref_lib() is not None else "port"
    ck = CheckerScene(desc, "ref" if kind == "reference" else "oracle")
    img = np.zeros((len(px), 3), np.float32)
    refc, done, t_ref = [], 0, 0.0
    for spp in cfg["SPP"]:
        t1 = time.perf_counter()
        img, _ = ck.pathtrace(cam.flat(), W, H, done, spp - done, D, pixels=px, img=img, threads=threads)
        t_ref += time.perf_counter() - t1
        done = spp
        refc.append(rmse(img))
    ref_mpaths = len(px) * done / t_ref / 1e6
    # the GPU ground truth of the cache line (1024 spp, frames 2^21 ..) against the FP64 render
    r.set_method(cb.RenderingMethod.PATHTRACER)  # clears the image
    r.set_frame_index(1 << 21)
    r.render_frames(cam, 1024)
    g = r.get_output_image().numpy().reshape(-1, 3)[px].astype(np.float64) * ((1 << 21) + 1024) / 1024
    rel = float(np.abs(g - gt).sum() / max(np.abs(gt).sum(), 1e-30))
    line = {"metric": cfg["metric"], "value": ours_mpaths, "unit": "Mpaths/s", "n_gpus": 1, "steps": 64,
            "warmup": args.warmup, "ms_per_step": W * H / (ours_mpaths * 1e6) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "width": W, "height": H, "max_trace_depth": D,
                       "pixels": len(px), "ground_truth_spp": n, "ground_truth_s": round(t_gt, 1),
                       "threads": threads},
            "equal_rmse": {"spp": list(cfg["SPP"]), "rmse_this_library": ours, "rmse_reference_host": refc,
                           "curves_equal": bool(np.allclose(ours, refc, rtol=1e-3)),
                           "note": "equal RMSE at equal spp: Mpaths/s at equal RMSE is each arm's Mpaths/s"},
            "reference_host": {"value": ref_mpaths, "unit": "Mpaths/s", "kind": kind, "cores": threads,
                               "sample": f"{len(px)} pixels x {done} spp"},
            "cache_ground_truth_check": {"gpu_spp": 1024, "relative_l1_vs_fp64": rel,
                                         "note": "the radiance-cache line's GPU ground truth at these pixels "
                                                 "against the FP64 oracle render"}}
    print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def _median(v):
    v = sorted(v)
    return v[len(v) // 2]


def run_method(args) -> int:
    """VOLUME or GRADIENTDOMAIN (RenderingMethod) on its scene: the median of
    5 timed regions of `steps` render() calls each, a byte-model roofline
    from an instrumented frame's traversal counts, the reference's CUDA
    build timed on the same GPU and its host build on the CPU cores."""
    import numpy as np
    import torch
    import cupbr_b200 as cb
    from cupbr_b200 import scenes

    cfg = SCENES[args.scene]
    W, H, DEPTH = cfg["W"], cfg["H"], cfg["DEPTH"]
    method = cb.RenderingMethod.VOLUME if args.scene == "volume" else cb.RenderingMethod.GRADIENTDOMAIN
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)
    desc = scenes.volume_test_scene() if args.scene == "volume" else scenes.cornell_box()
    sc = desc.build()
    stream = torch.cuda.Stream()
    r = cb.PBRenderer(method)
    r.set_output_size(W, H)
    r.register_scene(sc)
    r.set_method(method)
    r.set_max_trace_depth(DEPTH)
    r.set_russian_roulette(False)
    r.set_stream(stream)
    cam = cb.Camera(W, H)
    r.set_frame_index(frame_base(rank))
    r.set_instrumented(True)
    r.render(cam)
    st = r.stats()
    r.set_instrumented(False)
    sampler = ClockSampler(local)
    # the `steps` frames of a timed region through one render_frames() call:
    # multi-frame wavefronts (VOLUME; GDPT: the paths, each frame's running
    # means and 50-pass reconstruction still in order), the images of one
    # render() per frame
    batched = True
    for _ in range(args.warmup):
        r.render(cam)
    if batched:
        r.render_frames(cam, args.steps)  # allocates the multi-frame workspace outside the timed regions
    torch.cuda.synchronize()
    sampler.settle()
    if world > 1:
        torch.distributed.barrier()
    times = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if batched:
            r.render_frames(cam, args.steps)
        else:
            for _ in range(args.steps):
                r.render(cam)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = _median(times)
    # the GDPT reconstruction alone on the renderer's own buffers (51 launches per step)
    rec_ms = None
    if args.scene == "gdpt":
        n = W * H
        bufs = [torch.zeros((n, 3), device="cuda") for _ in range(9)]
        cb._native.call("cupbr_gdpt_reconstruct", W, H, *[b.data_ptr() for b in bufs[:5]],
                        *[b.data_ptr() for b in bufs[5:]], stream.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            cb._native.call("cupbr_gdpt_reconstruct", W, H, *[b.data_ptr() for b in bufs[:5]],
                            *[b.data_ptr() for b in bufs[5:]], stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        rec_ms = e0.elapsed_time(e1)
    # end to end: one render() with the camera from host memory + HDR readback
    # per step, render() pipelined as in the path tracer's e2e line
    host = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True)
    img = r.get_output_image()
    r.set_pipelined(True)
    for _ in range(4):  # each internal stream's workspace, outside the timed region
        r.render(cam)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        r.render(cam)
        cb._native.call("cupbr_memcpy_d2h", host.data_ptr(), img.ptr, img.nbytes, stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    ms, ms_e2e = max_over_ranks([ms, ms_e2e])
    samples = W * H * args.steps * world
    value = samples / (ms * 1e-3) / 1e6
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    # traversal bytes of one frame on the path tracer's model (node 112 B,
    # triangle 48 B, 96 B of ray state per ray) + 12 B per image write / pixel
    # (GDPT: 5 running means of 12 B read and written)
    rays = st["ext_rays"] + st["shadow_rays"]
    frame_bytes = (112.0 * (st["ext_nodes"] + st["shadow_nodes"]) + 48.0 * (st["ext_prims"] + st["shadow_prims"])
                   + 96.0 * rays + (24.0 if args.scene == "volume" else 120.0) * W * H)
    path_ms = ms - (rec_ms or 0.0)
    achieved = frame_bytes * args.steps / (path_ms * 1e-3) / 1e9
    if rank == 0:
        kname = ("VOLUME wavefront frame: k_extend_camera / k_extend, k_vol_shade, k_connect per depth"
                 if args.scene == "volume" else
                 "GDPT wavefronts (base paths, then shift paths): k_extend_camera / k_extend, k_gd_shade, k_connect "
                 "per depth")
        line = {"metric": cfg["metric"], "value": value, "unit": "Mpaths/s" if args.scene == "volume" else
                "Mpixel-samples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": cfg["workload"], "width": W, "height": H, "max_trace_depth": DEPTH,
                           "l2": cfg["l2"], "parallelism": f"replicas{world}",
                           "timing": "median of 5 timed regions of `steps` frames (" +
                                     ("one render_frames() call" if batched else "render() per frame") + ")"},
                "repeats_ms": times,
                "e2e": {"value": samples / (ms_e2e * 1e-3) / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step":
                        cb._native.C.sizeof(cb._native.Camera), "d2h_bytes_per_step": W * H * 12,
                        "note": "one render() + HDR readback per step (render() pipelined)"},
                "rays_per_frame": {"closest": st["ext_rays"], "occlusion": st["shadow_rays"]},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "traffic": None, "peak_source": f"{peak_src} hbm_gbs", "kernel": kname,
                             "bytes_model": "112*node_visits + 48*triangle_tests + 96 per ray + image writes, "
                                            "from an instrumented frame; the scene is L2-resident, so the "
                                            "fraction says how fast the kernel consumes the algorithm's reads",
                             "bytes_per_step": frame_bytes},
                "gpu_launches": ((2 + 3 * DEPTH) * -(-args.steps // max(1, BATCH_PATHS // (W * H)))
                                 if args.scene == "volume" else
                                 2 * (1 + 3 * DEPTH) * -(-args.steps // max(1, BATCH_PATHS // (5 * W * H)))
                                 + 52 * args.steps),
                "device_errors": r.error_count(), "clocks": clocks}
        if rec_ms is not None:
            rec_bytes = 72.0 * W * H * 50 + 72.0 * W * H  # 50 passes of 5 reads + 1 write, init 6 reads + 3 writes
            line["roofline_reconstruction"] = {
                "kernel": "k_gdpt_init + 10 x k_gdpt_opt_blocked (5 passes each)", "ms_per_step": rec_ms / args.steps,
                "achieved": rec_bytes * args.steps / (rec_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                "frac": rec_bytes * args.steps / (rec_ms * 1e-3) / 1e9 / peak,
                "note": "algorithmic 72 B per pixel and pass (50 passes); the blocked kernel reads each image once per 5 passes, and the nine 3 MB images stay in L2"}
        if world == 1 and not args.no_reference_cuda:
            try:
                from oracle import bridge
                if bridge.ref_cuda_lib() is not None:
                    rs = bridge.RefCudaScene(desc)
                    fn = rs.volumetrace if args.scene == "volume" else rs.gradientdomain
                    fn(cam.flat(), W, H, 0, 1, DEPTH)
                    _, rms = fn(cam.flat(), W, H, 0, args.steps, DEPTH)
                    line["reference_cuda"] = {"value": W * H * args.steps / (rms * 1e-3) / 1e6,
                                              "unit": line["unit"], "ms": rms,
                                              "kind": "reference PBRendering::" + ("volumetracing" if args.scene ==
                                                                                  "volume" else "gradientdomain") +
                                                      ", sm_100a, -use_fast_math, same GPU",
                                              "speedup_of_value": value / (W * H * args.steps / (rms * 1e-3) / 1e6)}
            except Exception as exc:
                line["reference_cuda"] = {"unavailable": str(exc)[:200]}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = method_cpu_sample(desc, args.scene, DEPTH)
        print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def method_cpu_sample(desc, scene, depth):
    """The reference's host build (or the oracle) on a 128x128 frame of the
    same scene and method."""
    import numpy as np
    from oracle.bridge import CheckerScene, ref_lib
    kind = "reference" if ref_lib() is not None else "port"
    sc = CheckerScene(desc, "ref" if kind == "reference" else "oracle")
    w = h = 128
    aspect = np.float32(w) / np.float32(h)
    cam = np.array([0, 0, 0, aspect, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < 5.0:
        if scene == "volume":
            sc.volumetrace(cam, w, h, n, 1, depth)
        else:
            sc.gdpt(cam, w, h, n, 1, depth)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": w * h * n / dt / 1e6, "unit": "Mpaths/s" if scene == "volume" else "Mpixel-samples/s",
            "cores": 1, "kind": kind, "sample": f"{n} frames of {w}x{h}, one host thread, {dt:.1f} s"}


def run_post(args) -> int:
    """Bloom + tone map (PostProcessor::bloom, ToneMapper::toneMap) of a
    7680x4320 HDR image: the fused two-kernel pass, the median of 5 timed
    regions of `steps` passes, against the reference's CUDA build."""
    import numpy as np
    import torch
    import cupbr_b200 as cb

    cfg = SCENES["post"]
    W, H = cfg["W"], cfg["H"]
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)
    rng = np.random.default_rng(9)
    hdr_host = ((rng.random((H, W, 3), dtype=np.float32) * 2.0) ** 3).astype(np.float32)
    hdr = torch.from_numpy(hdr_host).cuda()
    stream = torch.cuda.Stream()
    pp = cb.PostProcessor()
    pp.set_stream(stream)
    pp.register_image(cb.DeviceImage(hdr.data_ptr(), W, H, 3, np.float32, owner=hdr))
    rgba = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    out = cb.DeviceImage(rgba.data_ptr(), W, H, 4, np.uint8, owner=rgba)
    th = cb.threshold_curve(1.0, 1.0)
    sampler = ClockSampler(local)
    for _ in range(args.warmup):
        pp.bloom_tonemap(th, cb.ToneMappingType.REINHARD, 1.0, out)
    torch.cuda.synchronize()
    sampler.settle()
    times = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            pp.bloom_tonemap(th, cb.ToneMappingType.REINHARD, 1.0, out)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = _median(times)
    # end to end: HDR image from pinned host memory, RGBA8 back, per step
    hp = torch.from_numpy(hdr_host).pin_memory()
    ho = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        cb._native.call("cupbr_memcpy_h2d", hdr.data_ptr(), hp.data_ptr(), hdr.numel() * 4, stream.cuda_stream)
        pp.bloom_tonemap(th, cb.ToneMappingType.REINHARD, 1.0, out)
        cb._native.call("cupbr_memcpy_d2h", ho.data_ptr(), rgba.data_ptr(), rgba.numel(), stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    ms, ms_e2e = max_over_ranks([ms, ms_e2e])
    px = W * H * args.steps * world
    value = px / (ms * 1e-3) / 1e6
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    # k_bloom_down: 12 B read + 3 B written per pixel (half resolution);
    # k_bloom_up fused with the tone map: 12 + 3 B read, 4 B written
    bytes_px = 12.0 + 3.0 + 12.0 + 3.0 + 4.0
    achieved = bytes_px * W * H * args.steps / (ms * 1e-3) / 1e9
    if rank == 0:
        line = {"metric": cfg["metric"], "value": value, "unit": "Mpixels/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": cfg["workload"], "width": W, "height": H, "l2": cfg["l2"],
                           "parallelism": f"replicas{world}",
                           "timing": "median of 5 timed regions of `steps` passes"},
                "repeats_ms": times,
                "e2e": {"value": px / (ms_e2e * 1e-3) / 1e6, "unit": "Mpixels/s",
                        "h2d_bytes_per_step": hdr.numel() * 4, "d2h_bytes_per_step": rgba.numel(),
                        "note": "HDR upload + bloom/tone map + RGBA8 readback per step"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "peak_source": f"{peak_src} hbm_gbs",
                             "kernel": "k_bloom_down + k_bloom_up (fused tone map)", "bytes_per_pixel": bytes_px},
                "gpu_launches": 2 * args.steps, "clocks": clocks}
        if world == 1 and not args.no_reference_cuda:
            try:
                from oracle import bridge
                if bridge.ref_cuda_lib() is not None:
                    b_ms, t_ms = bridge.ref_cuda_post_timed(hdr_host, th, 0, 1.0, iters=max(1, min(args.steps, 5)))
                    line["reference_cuda"] = {"value": W * H / ((b_ms + t_ms) * 1e-3) / 1e6, "unit": "Mpixels/s",
                                              "ms_bloom": b_ms, "ms_tonemap": t_ms,
                                              "kind": "reference PostProcessor::bloom + ToneMapper::toneMap, sm_100a, "
                                                      "-use_fast_math, same GPU",
                                              "speedup_of_value": value / (W * H / ((b_ms + t_ms) * 1e-3) / 1e6)}
            except Exception as exc:
                line["reference_cuda"] = {"unavailable": str(exc)[:200]}
        if world == 1 and not args.no_cpu_baseline:
            # the oracle's restatement of PostProcessor::bloom + ToneMapper::toneMap
            # (one host thread) on a 1920x1080 crop of the same image
            from oracle import bridge
            crop = np.ascontiguousarray(hdr_host[:1080, :1920])
            reps, t0 = 0, time.perf_counter()
            while reps < 1 or time.perf_counter() - t0 < 5.0:
                bridge.tonemap(bridge.bloom(crop, np.asarray(th, np.float32)), 0, 1.0)
                reps += 1
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": 1920 * 1080 * reps / dt / 1e6, "unit": "Mpixels/s", "cores": 1,
                                    "kind": "port",
                                    "sample": f"{reps} passes over a 1920x1080 crop of the image, oracle bloom + "
                                              f"Reinhard tone map, 1 thread, {dt:.1f} s"}
        print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def run_cache(args) -> int:
    """Radiance cache against plain NEE path tracing at equal device time.

    Ground truth: GT_SPP plain samples per pixel in two disjoint halves, whose
    difference estimates the ground truth's own variance, which is taken out
    of both MSEs.  Plain arm: `steps` frames (the time budget).  Cached arm:
    a cache trained for CACHE_WARMUP frames (time reported as warm-up), then
    as many cached frames, with online training, as fit in the plain arm's
    device time."""
    import numpy as np
    import torch
    import cupbr_b200 as cb
    from cupbr_b200.cache import RadianceCache

    cfg = SCENES["cache"]
    W, H, D = cfg["W"], cfg["H"], cfg["DEPTH"]
    world, rank, local = init_replicas()
    torch.cuda.set_device(local)
    desc = make_scene("cache")
    sc = desc.build()
    info = sc.info()
    stream = torch.cuda.Stream()
    cam = cb.Camera(W, H)
    K = args.steps
    base = frame_base(rank)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    rp = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    rp.set_output_size(W, H)
    rp.register_scene(sc)
    rp.set_method(cb.RenderingMethod.PATHTRACER)
    rp.set_max_trace_depth(D)
    rp.set_russian_roulette(False)
    rp.set_stream(stream)
    rp.set_pipelined(True)  # the plain arm at its fastest: overlapped wavefronts of the default size
    rp.set_batch_paths(BATCH_PATHS)
    rp.set_frame_index(base + (1 << 25))
    # allocates the wavefront buffers (a full wavefront) outside every timed region
    rp.render_frames(cam, max(args.warmup, BATCH_PATHS // (W * H)))

    plain_out = torch.as_tensor(rp.get_output_image(), device="cuda")

    def plain(frame0, frames):
        r = rp
        plain_out.zero_()  # a mean started at frame0 > 0 accumulates onto the image
        r.set_frame_index(frame0)
        e0, e1 = ev(), ev()
        torch.cuda.synchronize()
        e0.record(stream)
        r.render_frames(cam, frames)
        e1.record(stream)
        torch.cuda.synchronize()
        # a running mean started at frame0 > 0 from zero holds sum / (frame0 + frames)
        img = r.get_output_image().numpy().astype(np.float64) * ((frame0 + frames) / frames)
        return img, e0.elapsed_time(e1), r

    half = cfg["GT_SPP"] // 2
    ga, t_gt, _ = plain(base + (1 << 24), half)
    gb, _, _ = plain(base + (1 << 24) + (1 << 20), half)
    gt = 0.5 * (ga + gb)
    var_gt = float(((ga - gb) ** 2).mean() / 4.0)
    del ga, gb

    def mse(img):
        return float(((np.asarray(img, np.float64) - gt) ** 2).mean()) - var_gt

    sampler = ClockSampler(local)
    cache = RadianceCache(sc, cache_depth=cfg["CACHE_DEPTH"], train_stride=cfg["TRAIN_STRIDE"],
                          learning_rate=cfg["LR"])
    if args.cache_batch_paths:
        cache.set_batch_paths(args.cache_batch_paths)
    scratch = torch.zeros((H, W, 3), device="cuda")
    e0, e1 = ev(), ev()
    torch.cuda.synchronize()
    e0.record(stream)
    cache.render(sc, cam, W, H, base + (1 << 22), cfg["CACHE_WARMUP"], D, scratch.data_ptr(), train=True,
                 stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    warm_ms = e0.elapsed_time(e1)
    # per-frame time of the cached renderer with training (for the equal-time frame count)
    e0.record(stream)
    cache.render(sc, cam, W, H, base + (1 << 22) + 4096, 8, D, scratch.data_ptr(), train=True,
                 stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_cached_frame = e0.elapsed_time(e1) / 8
    sampler.settle()
    if world > 1:
        torch.distributed.barrier()

    rows = []
    budgets = sorted({4, K, 64}) if world == 1 else [K]
    main = None
    for B in budgets:
        p_img, t_plain, _ = plain(base, B)
        n = max(1, int(t_plain / t_cached_frame))
        img = torch.zeros((H, W, 3), device="cuda")
        if B == K:
            cache.set_profiling(True)
        e0.record(stream)
        cache.render(sc, cam, W, H, base, n, D, img.data_ptr(), train=True, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t_cached = e0.elapsed_time(e1)
        row = {"plain_frames": B, "plain_ms": round(t_plain, 3), "plain_mse": mse(p_img), "cached_frames": n,
               "cached_ms": round(t_cached, 3), "cached_mse": mse(img.cpu().numpy())}
        row["mse_ratio"] = row["plain_mse"] / row["cached_mse"]
        if B == K:
            stages, waves = cache.stage_times()
            cache.set_profiling(False)
            main = (row, stages, waves, n, t_cached, t_plain)
        rows.append(row)
    clocks = sampler.stop()
    row, stages, waves, n, t_cached, t_plain = main
    t_cached, t_plain = max_over_ranks([t_cached, t_plain])
    errors = cache.counters()[0]

    # one profiled wavefront of the cache's wavefront size: inference and
    # training work and time for the roofline
    cache.set_profiling(True)
    frames_per_wave = max(1, min(n, (args.cache_batch_paths or CACHE_BATCH_PATHS) // (W * H)))
    cache.render(sc, cam, W, H, base + (1 << 21), frames_per_wave, D, scratch.data_ptr(), train=True,
                 stream=stream.cuda_stream)
    torch.cuda.synchronize()
    st1, _ = cache.stage_times()
    cache.set_profiling(False)
    _, queries, samples = cache.counters()
    steps_per_wave = frames_per_wave * (cache.desc.samples_per_frame // cache.desc.batch)
    infer_flop = 2 * (96 * 64 + 4 * 64 * 64 + 64 * 3)  # per query (16 output rows computed, 3 used)
    train_flop = 3 * infer_flop                            # forward + input and weight gradients per sample
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 1590.0, "fallback"
    if os.path.exists(peaks_path):
        peak, peak_src = float(json.load(open(peaks_path))["bf16_tflops"]), "measured"
    achieved = infer_flop * queries / (st1["infer"] * 1e-3) / 1e12 if st1["infer"] > 0 else 0.0
    train_tflops = (train_flop * cache.desc.batch * steps_per_wave / (st1["train"] * 1e-3) / 1e12
                    if st1["train"] > 0 else 0.0)
    traffic = NCU_TRAFFIC["k_rc_infer heightfield"]["bytes_per_query"]

    # end to end through the public API: each step renders E2E_FRAMES frames,
    # tone maps them and reads the RGBA8 frame back to pinned host memory
    FE = cfg["E2E_FRAMES"]
    rgba = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    host = torch.empty(rgba.numel(), dtype=torch.uint8, pin_memory=True)
    r_e2e = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r_e2e.set_output_size(W, H)
    r_e2e.register_scene(sc)
    r_e2e.set_method(cb.RenderingMethod.PATHTRACER)
    r_e2e.set_max_trace_depth(D)
    r_e2e.set_russian_roulette(False)
    r_e2e.set_stream(stream)
    r_e2e.set_frame_index(base)
    out = r_e2e.get_output_image()

    def readback(ptr):
        cb._native.call("cupbr_tonemap", ptr, W, H, 0, 1.0, rgba.data_ptr(), stream.cuda_stream)
        cb._native.call("cupbr_memcpy_d2h", host.data_ptr(), rgba.data_ptr(), rgba.numel(), stream.cuda_stream)

    steps_plain = max(1, K // FE)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps_plain):
        r_e2e.render_frames(cam, FE)
        readback(out.ptr)
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain_e2e = e0.elapsed_time(e1)
    mse_plain_e2e = mse(out.numpy())
    img = torch.zeros((H, W, 3), device="cuda")
    # per-step time of the cached arm, then as many steps as fit in the plain arm's time
    e0.record(stream)
    for i in range(4):
        cache.render(sc, cam, W, H, base + (1 << 20) + FE * i, FE, D, scratch.data_ptr(), train=True,
                     stream=stream.cuda_stream)
        readback(scratch.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    steps_cached = max(1, int(t_plain_e2e / (e0.elapsed_time(e1) / 4)))
    e0.record(stream)
    for i in range(steps_cached):
        cache.render(sc, cam, W, H, base + FE * i, FE, D, img.data_ptr(), train=True, stream=stream.cuda_stream)
        readback(img.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    t_cached_e2e = e0.elapsed_time(e1)
    e2e_ratio = mse_plain_e2e / mse(img.cpu().numpy())
    cam_bytes = cb._native.C.sizeof(cb._native.Camera)

    if rank == 0:
        launches_per_wave = 1 + 3 * D + 1 + 1 + 1 + 2 * steps_per_wave
        config = {"workload": cfg["workload"], "width": W, "height": H, "max_trace_depth": D,
                  "russian_roulette": False, "l2": cfg["l2"], "data": "synthetic, seed 0",
                  "parallelism": f"replicas{world}", "triangles": info["triangles"],
                  "cache_depth": cfg["CACHE_DEPTH"], "train_stride": cfg["TRAIN_STRIDE"], "learning_rate": cfg["LR"],
                  "loss": "relative L2", "cache_warmup_frames": cfg["CACHE_WARMUP"],
                  "ground_truth": f"plain path tracer, {cfg['GT_SPP']} spp in two halves; their variance "
                                  f"({var_gt:.3e}) is subtracted from both MSEs",
                  "frames_per_wavefront": frames_per_wave}
        line = {"metric": cfg["metric"], "value": row["mse_ratio"], "unit": "x", "n_gpus": world, "steps": K,
                "warmup": args.warmup, "ms_per_step": t_plain / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 tracing, f16 MLP with f32 accumulation", "data": "synthetic",
                "config": config,
                "equal_time": row, "budgets": rows,
                "cached_mpaths_per_s": W * H * n * world / (t_cached * 1e-3) / 1e6,
                "plain_mpaths_per_s": W * H * K * world / (t_plain * 1e-3) / 1e6,
                "cache_warmup_ms": warm_ms,
                "stage_ms_per_cached_frame": {k: round(v / n, 4) for k, v in stages.items()},
                "e2e": {"value": e2e_ratio, "unit": "x", "h2d_bytes_per_step": cam_bytes,
                        "d2h_bytes_per_step": rgba.numel(),
                        "note": f"each step renders {FE} frames, tone maps and reads the RGBA8 frame back; "
                                f"plain {steps_plain} steps in {t_plain_e2e:.1f} ms, cached {steps_cached} steps in "
                                f"{t_cached_e2e:.1f} ms"},
                "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                             "frac": achieved / peak, "traffic": (traffic * queries) if traffic else None,
                             "peak_source": f"{peak_src} bf16_tflops (dense f16 runs at the bf16 rate)",
                             "kernel": "k_rc_infer (cache queries of one wavefront)",
                             "flop_per_launch": infer_flop * queries, "queries": queries,
                             "flop_model": "2*(96*64 + 4*64*64 + 64*3) = 45,440 per query"},
                "training": {"tflops": train_tflops, "samples_per_step": cache.desc.batch,
                             "steps_per_wavefront": steps_per_wave, "samples_collected": samples,
                             "flop_model": "3 x 45,440 per sample (forward, input and weight gradients)"},
                "gpu_launches": waves * launches_per_wave,
                "device_errors": errors,
                "clocks": clocks}
        if world == 1 and not args.no_cpu_baseline:
            v, kind, sample = cpu_reference_sample(desc, SCENES["heightfield"], args.cpu_seconds,
                                                   os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": v, "unit": "Mpaths/s (plain path tracing)", "cores": os.cpu_count() or 1,
                                    "kind": kind, "sample": sample}
        print(json.dumps(line), flush=True)
    finish_replicas()
    return 0


def main() -> int:
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="default: 256 frames (path tracer), 128 spp (medium), 2 batch launches (batch), "
                         "16 plain frames of time budget (cache)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scene", default="heightfield", choices=sorted(SCENES))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--reference-seconds", type=float, default=60.0)
    ap.add_argument("--no-fd-check", action="store_true")
    ap.add_argument("--repeats", type=int, default=None,
                    help="timed regions of K steps whose median is the value (default 1; 5 for --scene cornell)")
    ap.add_argument("--cache-batch-paths", type=int, default=0,
                    help="paths per cached wavefront (--scene cache; 0: the library default)")
    ap.add_argument("--resolution", default=None,
                    help="WxH override of the workload's image size (small cases for profiling)")
    ap.add_argument("--batch-paths", type=int, default=0,
                    help="override of the path tracer's paths per wavefront (small device footprints for profiling)")
    args = ap.parse_args()
    if args.batch_paths:
        global BATCH_PATHS
        BATCH_PATHS = args.batch_paths
    if args.resolution:
        w, h = (int(v) for v in args.resolution.lower().split("x"))
        for cfg in SCENES.values():
            if cfg["W"]:
                cfg["W"], cfg["H"] = w, h
                cfg["workload"] += f" [image size overridden to {w}x{h}]"
    if args.repeats is None:
        args.repeats = 5 if args.scene in ("cornell", "medium") else 1
    if args.steps is None:
        args.steps = {"cornell": 8192}.get(args.scene) or {"batch": 2, "medium": 2048, "cache": 16, "volume": 64, "gdpt": 32, "post": 10}.get(args.scene, 256)
    if args.scene == "cache":
        if args.impl == "reference":
            if _dist()[1] == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no radiance cache "
                                  "(its path tracer, PathTracer.cu, traces every path to the end)"}), flush=True)
            return 0
        return run_cache(args)
    if args.scene == "batch":
        if args.impl == "reference":
            return run_reference_batch(args)
        return run_batch(args)
    if args.scene == "rmse":
        if args.impl == "reference":
            if _dist()[1] == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference's host build is the second "
                                  "curve of the b200 line (equal_rmse)"}), flush=True)
            return 0
        return run_rmse(args)
    if args.scene in ("volume", "gdpt", "post"):
        if args.impl == "reference":
            if _dist()[1] == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference's CUDA build is timed inside "
                                  "the b200 line (reference_cuda) for this workload"}), flush=True)
            return 0
        return run_post(args) if args.scene == "post" else run_method(args)
    if args.scene == "medium":
        if args.impl == "reference":
            if _dist()[1] == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no density-grid medium "
                                  "(VolumeRenderer.cu renders homogeneous media only)"}), flush=True)
            return 0
        return run_medium(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
