"""Benchmark: phiray's Rendered-mode hot path on the B200.

Workload (the single-large-mesh configuration): an icosphere subdivided 8
times (1,310,720 faces) displaced by seeded value noise, a ground plane, 4
area lights, 30% mirror faces, 1920 x 1080, 64 samples per pixel, 8 diffuse
bounces. One step is one frame: the LBVH rebuilt on the device over the
mesh's face boxes, 64 samples traced, the a-trous denoise. Inputs are
seeded synthetic (no dataset exists for this path).

The headline `value` is Mrays/s over the whole frame step (every closest-hit
and shadow ray the path tracer traced), whole job over all ranks. `e2e` is
the same metric through the public API from pinned host arrays: create the
tracer (scene upload + build), trace, denoise, read the packed image back.

`--impl reference` times the reference's algorithm on the host cores (the
C++ restatement of phiray's CPU twins and WGSL, oracle/, OpenMP over every
core) on a bounded sample of the same frame.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1080p frames/s at equal relMSE vs 4096spp: denoised low-spp vs plain; Mrays/s"
UNIT = "Mrays/s"
WORKLOAD = ("c2_mesh: icosphere L8 (1,310,722 tris) + 4 area lights, 1920x1080, 64 spp, 8 bounces, "
            "tree rebuild (the autotuner's pick of LBVH or binned SAH) + trace + denoise per frame")


KERNEL_NAMES = ["megakernel", "state-machine/4", "state-machine/6", "state-machine/8", "megakernel/3", "megakernel/2",
                "megakernel/sync", "megakernel/2/sync", "megakernel/5", "megakernel/6", "megakernel/6/sync", "megakernel/8", "megakernel/8/sync",
                "megakernel/10/sync", "megakernel/12/sync", "megakernel/16/sync", "wavefront",
                "megakernel/reg8", "megakernel/8/sync/reg1", "megakernel/16/sync/reg1"]


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class Clocks:
    """nvidia-smi samples during the timed region (median SM clock, reasons)."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[2:]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float, device: str = "cuda") -> float:
    """The largest `value` over all ranks of the default process group (the
    timing rule: a multi-GPU step takes as long as its slowest rank); the
    value itself when there is no group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, ms_max: float) -> float:
    """Whole-job throughput of replicas: every rank processes `units_per_rank`
    in (at most) ms_max milliseconds."""
    return units_per_rank * world / (ms_max * 1e-3)


# The c2 frame's shape, printed identically by both arms.
C2_CONFIG = {"workload": WORKLOAD, "frame": "1920x1080", "spp": 64, "bounces": 8, "tris": 1310722}
SAMPLE_ROWS = 48  # rows of the CPU legs' stratified sample


def sample_rows(h: int, k: int = SAMPLE_ROWS, seed: int = 0x2545F491) -> list[int]:
    """One row from each of k equal strata of an h-row frame, at a seeded
    offset inside its stratum: the CPU legs' bounded, frame-wide sample
    (both arms trace the same rows)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    edges = np.linspace(0, h, k + 1)
    return [int(min(h - 1, np.floor(edges[i] + rng.random() * (edges[i + 1] - edges[i])))) for i in range(k)]


def trace_sample(T, cam, px, rows) -> tuple[int, float]:
    """The oracle over the sample rows at 1 spp: (rays, seconds)."""
    rays_total, t_total = 0, 0.0
    for r in rows:
        t0 = time.perf_counter()
        _, rays = T.trace(cam, 0, 1, px, rows=(r, 1))
        t_total += time.perf_counter() - t0
        rays_total += rays
    return rays_total, t_total


def reference_arm(args) -> None:
    """The reference's algorithm on the host cores (the oracle restatement)."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from phiray_b200 import scenes
    from phiray_b200.tracer import camera
    from tests import oracle_lib

    orc = oracle_lib.load()
    threads = orc.lib.orc_threads()
    s = scenes.c2_mesh()
    cam = camera(s)
    cam["w"], cam["h"] = s.width, s.height
    # the binned SAH tree phiray's tracer walks (sah.rs), built once outside the timing
    T = oracle_lib.TraceOracle(orc, s, sah=True)
    px = np.zeros(34 * s.width * s.height + 1, np.uint32)
    rows = sample_rows(s.height)  # a bounded sample: one seeded row from each of 48 strata, one sample each
    vals = []
    for k in range(args.warmup + args.steps):
        rays, dt = trace_sample(T, cam, px, rows)
        if k >= args.warmup:
            vals.append(rays / dt / 1e6)
    v = statistics.median(vals)
    line = {
        "metric": METRIC, "value": round(v, 3), "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": dict(C2_CONFIG),
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(rows)} rows of the 1080p frame (one seeded row a stratum) at 1 spp per "
                                   "step over the SAH tree (oracle/ C++ restatement, OpenMP)"},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(scene, cam) -> dict:
    """The oracle traced on the host cores over a bounded sample (~10 s)."""
    from tests import oracle_lib

    orc = oracle_lib.load()
    T = oracle_lib.TraceOracle(orc, scene, sah=True)  # phiray's tracer walks the SAH tree (sah.rs)
    px = np.zeros(34 * scene.width * scene.height + 1, np.uint32)
    rows = sample_rows(scene.height)  # the reference arm's sample
    rays_total, t_total, passes = 0, 0.0, 0
    while t_total < 10.0 and passes < 20:
        rays, dt = trace_sample(T, cam, px, rows)
        rays_total += rays
        t_total += dt
        passes += 1
    return {"value": round(rays_total / t_total / 1e6, 3), "unit": UNIT, "cores": orc.lib.orc_threads(), "kind": "port",
            "sample": f"{passes} x {len(rows)} rows of the 1080p frame (one seeded row a stratum, the reference "
                      f"arm's sample) at 1 spp over the SAH tree ({rays_total} rays, {t_total:.1f} s), "
                      "oracle/ C++ OpenMP"}


def profile_phase(args, tr, gpu, cam, verts_dev, W, H, n, local) -> None:
    """Warm-up and steps of one kernel family alone (for ncu launch lists and
    captures): the frame render, the incoherent ray walk, or the LBVH build."""
    import torch

    if args.phase == "render":
        if args.kernel >= 0:
            tr.set_kernel(args.kernel)
        if args.adapt:
            thr, lo, step = (float(v) for v in args.adapt.split(","))
            tr.set_adaptive([thr, lo, step, 1.0])
        fn = lambda: tr.trace(cam, W, H, 0, args.spp)  # noqa: E731
    elif args.phase == "build":
        fn = lambda: tr.repose_device(verts_dev, rebuild=True)  # noqa: E731
    else:
        rays = torch.empty((n, 8), dtype=torch.float32, device=f"cuda:{local}")
        hits = torch.empty((n, 4), dtype=torch.float32, device=f"cuda:{local}")
        tr.secondary_rays(cam, W, H, 0, rays)
        tr.set_walk(args.walk)
        tr.set_stack(args.stack)
        fn = lambda: tr.trace_rays(rays, n, hits, False)  # noqa: E731
    for _ in range(args.warmup):
        fn()
    gpu.wait(60000)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn()
    gpu.wait(60000)
    line = {"phase": args.phase, "steps": args.steps, "ms": (time.perf_counter() - t0) * 1e3 / args.steps}
    if args.phase == "render":
        gpu_ms, rays = tr.time()  # the last frame: device time and rays traced
        line.update({"gpu_ms": round(gpu_ms, 3), "rays": int(rays), "mrays_s": round(rays / gpu_ms / 1e3, 1)})
        if args.adapt:
            line["unconverged"] = tr.unconverged()
    print(json.dumps(line))


def run_c3(args) -> None:
    """The skinned-animation configuration: 500k vertices / ~1M faces, 64
    bones; per frame Skin -> face boxes -> LBVH refit (or full rebuild) ->
    trace 1080p at 16 spp, and the same on the binned SAH tree. Prints
    per-stage ms per frame (device events)."""
    import torch

    import phiray_b200 as px
    from phiray_b200 import scenes

    frames = args.frames
    s, rig = scenes.c3_skinned(spp=16)
    cam = px.camera(s)
    cam["w"], cam["h"] = s.width, s.height
    gpu = px.Gpu(0)
    st = torch.cuda.ExternalStream(gpu.stream)
    tr = px.Tracer.of(gpu, s)
    vptr, nv = tr.device_verts()
    dev = {k: torch.tensor(np.ascontiguousarray(a).view(np.uint8), device="cuda")
           for k, a in dict(rest=rig.rest, offsets=rig.offsets, pairs=rig.pairs).items()}
    bones = [torch.tensor(rig.bones(f), device="cuda") for f in range(frames)]
    gpu.wait(60000)
    torch.cuda.synchronize()
    # the render kernel for this scene, as the C2 leg picks it (same image)
    chosen, _ = tr.autotune(cam, s.width, s.height, 4)
    res = {}
    # the configuration's LBVH refit and rebuild, then the same over the
    # binned SAH tree (its Jacobi refit, its device rebuild)
    for mode in ("refit", "rebuild", "sah_refit", "sah_rebuild"):
        tr.set_tree(px.Tracer.TREE_SAH if mode.startswith("sah") else px.Tracer.TREE_LBVH)
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(frames)]
        rays = 0
        for f in range(frames + args.warmup):
            k = f - args.warmup
            e = ev[k] if k >= 0 else None
            if e:
                e[0].record(st)
            px.skin(gpu, dev["rest"], dev["offsets"], dev["pairs"], bones[f % frames], rig.nbones, vptr, nv, 1e-4)
            if e:
                e[1].record(st)
            tr.repose_device(vptr, rebuild=mode.endswith("rebuild"))
            if e:
                e[2].record(st)
            tr.trace(cam, s.width, s.height, 0, s.spp)
            if e:
                e[3].record(st)
            if k >= 0:
                rays += tr.time()[1] if k == 0 else 0
        gpu.wait(60000)
        torch.cuda.synchronize()
        skin = [e[0].elapsed_time(e[1]) for e in ev]
        bvh = [e[1].elapsed_time(e[2]) for e in ev]
        trace = [e[2].elapsed_time(e[3]) for e in ev]
        res[mode] = {"skin_ms": round(statistics.mean(skin), 3), "boxes_and_bvh_ms": round(statistics.mean(bvh), 3),
                     "trace_ms": round(statistics.mean(trace), 3),
                     "frame_ms": round(statistics.mean(skin) + statistics.mean(bvh) + statistics.mean(trace), 3)}
    nb = len(rig.rest)
    out = {"workload": "c3_skinned: 500k verts / 999k tris, 64 bones, 1-4 influences, 1080p 16 spp",
           "frames": frames, "per_frame": res, "render_kernel": KERNEL_NAMES[chosen],
           "skin_gbs": round((16 + 4 + 16 * len(rig.pairs) / nb + 16) * nb / (res["refit"]["skin_ms"] * 1e-3) / 1e9, 1)}
    print(json.dumps(out), flush=True)
    gpu.close()


def run_c4(args) -> None:
    """The learned denoiser's network alone: one forward pass over a 1080p
    frame (padded to 1088 x 1920) and one training step (forward, loss,
    backward, Adam) on `batch` 128 x 128 crops, timed with CUDA events on
    the context's stream; TFLOP/s counts the network's multiply-adds."""
    import torch

    import phiray_b200 as px
    from phiray_b200.denoiser import Unet, flops_per_pixel

    gpu = px.Gpu(0)
    stream = torch.cuda.ExternalStream(gpu.stream)
    net = Unet(gpu, seed=1)
    Hp, Wp, h, w = 1088, 1920, 1080, 1920
    g = torch.Generator(device="cpu").manual_seed(7)
    feat = (torch.randn(Hp, Wp, 16, generator=g) * 0.5).to(torch.bfloat16).cuda()
    irr = torch.rand(Hp, Wp, 3, generator=g).cuda()
    alb = (torch.rand(Hp, Wp, 3, generator=g) * 0.9 + 0.05).cuda()
    out = torch.empty(Hp, Wp, 3, device="cuda")
    err = torch.empty(Hp, Wp, device="cuda")
    torch.cuda.synchronize()

    def timed(fn, warm, reps):
        for _ in range(warm):
            fn()
        gpu.wait(60000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        gpu.wait(60000)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    fwd = lambda: net.forward(feat, irr, alb, 1, Hp, Wp, h, w, out, err)  # noqa: E731
    if args.phase == "nn":  # profiling runs: the launches alone
        for _ in range(args.warmup + args.steps):
            fwd()
        gpu.wait(60000)
        gpu.close()
        return
    with Clocks(0) as clk:
        fwd_ms = timed(fwd, args.warmup, args.steps)
    B, c = 12, 128
    tf = (torch.randn(B, c, c, 16, generator=g) * 0.5).to(torch.bfloat16).cuda()
    ti, ta = torch.rand(B, c, c, 3, generator=g).cuda(), (torch.rand(B, c, c, 3, generator=g) * 0.9 + 0.05).cuda()
    tref = torch.rand(B, c, c, 3, generator=g).cuda()
    loss = torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    step_ms = timed(lambda: net.train_step(tf, ti, ta, tref, B, c, c, c, c, loss, 1e-4), args.warmup, args.steps)
    fpp = flops_per_pixel()
    fwd_tflops = fpp * Hp * Wp / (fwd_ms * 1e-3) / 1e12
    train_tflops = 3 * fpp * B * c * c / (step_ms * 1e-3) / 1e12
    pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = pk.get("bf16_tflops", 1590.0)
    print(json.dumps({
        "metric": "learned denoiser network TFLOP/s (bf16 tensor cores, fp32 accumulate)",
        "value": round(fwd_tflops, 2), "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(fwd_ms, 3), "higher_is_better": True, "dtype": "bf16", "data": "synthetic",
        "config": {"workload": "KPCN U-Net 32-64-96-128-160, forward over 1088x1920; training step on 12 x 128^2",
                   "flops_per_pixel": fpp},
        "forward_ms": round(fwd_ms, 3), "train_step_ms": round(step_ms, 3), "train_tflops": round(train_tflops, 2),
        "roofline": {"bound": "tensor", "achieved": round(fwd_tflops, 2), "peak": peak, "unit": "TFLOP/s",
                     "frac": round(fwd_tflops / peak, 4), "peak_source": "measured" if pk else "fallback"},
        "clocks": clk.summary(),
    }), flush=True)
    net.close()
    gpu.close()


def run_c5(args) -> None:
    """Batched serving: 64 procedural scenes (10k-2M faces, 256^2 to 1080p,
    1/4/16 spp, 6 bounces) per frame: each scene's LBVH rebuilt or refit
    (seeded coin per scene per frame), every scene traced in one persistent
    launch, then the learned denoiser with its per-tile a-trous fallback;
    the whole frame is one captured CUDA graph, replayed per frame with the
    frame's rebuild/refit choices. Aggregate Mrays/s over the timed frames;
    per-scene latency = completion after the frame's start (device clock)."""
    import torch

    import phiray_b200 as px
    from phiray_b200 import scenes
    from phiray_b200.batch import Batch
    from phiray_b200.denoiser import THRESHOLD, WEIGHTS, Unet

    gpu = px.Gpu(0)
    stream = torch.cuda.ExternalStream(gpu.stream)
    t0 = time.time()
    scs = scenes.c5_batch(args.scenes)
    trs, b = [], Batch(gpu)
    for sc in scs:
        cam = px.camera(sc)
        cam["w"], cam["h"] = sc.width, sc.height
        tr = px.Tracer.of(gpu, sc)
        trs.append(tr)
        b.add(tr, cam, sc.width, sc.height, 0, sc.spp)
    setup_s = time.time() - t0
    cfg, tune_ms = b.autotune()
    net = Unet.pretrained(gpu) if os.path.exists(WEIGHTS) else Unet(gpu)
    b.capture(net, THRESHOLD)
    rng = np.random.default_rng(5)
    frames = [rng.integers(0, 2, len(scs)) for _ in range(args.warmup + args.steps)]
    for m in frames[:args.warmup]:
        b.replay(m)
    gpu.wait(60000)
    total_ms, rays, lats = 0.0, 0, []
    with Clocks(0) as clk:
        for m in frames[args.warmup:]:
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b.replay(m)
            e.record(stream)
            lat, r = b.results()
            torch.cuda.synchronize()
            total_ms += a.elapsed_time(e)
            rays += int(r.sum())
            lats.append(lat / 1e6)
    lats = np.concatenate(lats)
    ms = total_ms / args.steps
    value = rays / (total_ms * 1e-3) / 1e6
    print(json.dumps({
        "metric": "batched serving aggregate Mrays/s (64 scenes, one persistent launch, captured frame graph)",
        "value": round(value, 2), "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"c5_batch: {len(scs)} procedural scenes, faces log-uniform 10k-2M, "
                               "256^2/512^2/720p/1080p, 1/4/16 spp, 6 bounces, rebuild or refit per scene per frame, "
                               "learned denoise with a-trous fallback",
                   "faces_total": int(sum(sc.ntris for sc in scs)),
                   "pixels_total": int(sum(sc.width * sc.height for sc in scs)),
                   "samples_total": int(sum(sc.width * sc.height * sc.spp for sc in scs))},
        "frames_per_s": round(1000.0 / ms, 3),
        "latency_ms": {"p50": round(float(np.percentile(lats, 50)), 3),
                       "p99": round(float(np.percentile(lats, 99)), 3),
                       "max": round(float(lats.max()), 3)},
        "autotune": {"chosen": min(tune_ms, key=tune_ms.get), "kind_threads_stack": list(cfg),
                     "trace_ms": {k: round(v, 3) for k, v in tune_ms.items()}},
        "setup_s": round(setup_s, 1),
        "clocks": clk.summary(),
    }), flush=True)
    b.close()
    net.close()
    gpu.close()


def timed_fn(gpu, stream, fn, reps: int) -> float:
    """Mean device ms of fn over reps calls (after one untimed call), by
    CUDA events on the library's stream."""
    import torch

    fn()
    gpu.wait(60000)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    gpu.wait(60000)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def count_launches(fn) -> int:
    """Kernels one call of fn launches, counted by the CUDA activity trace
    of torch.profiler (every kernel of the process, the library's included)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    evs = [e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA and
           not e.name.startswith(("Memcpy", "Memset", "[memory]"))]
    return len(evs)


def equal_relmse(args, gpu, s, cam, stream, kernel: int = 0) -> dict:
    """The headline comparison at 1080p against a 4096-spp render of the same
    frame: plain tracing + the a-trous Denoise at `plain` spp against the
    learned denoiser (with its per-tile Denoise fallback) at `learned` spp.
    Every test image is an independent sample set: one accumulation runs the
    reference's 4096 samples first and each test image is the difference of
    two later accumulations (every plane the filters read accumulates
    linearly). relMSE = mean (x - r)^2 / (r^2 + 0.01) over pixels and
    channels of the linear mean over the samples that met something (the
    value the view transform shows; Tracer::radiance wherever every sample
    met something). Frame time = trace + filter, CUDA events."""
    import torch

    import phiray_b200 as px
    from phiray_b200 import kernels
    from phiray_b200 import train as T
    from phiray_b200.denoiser import THRESHOLD, TILE, WEIGHTS, Unet, snapshot_host

    if not os.path.exists(WEIGHTS):
        return {"unavailable": f"no trained weights at {os.path.relpath(WEIGHTS, ROOT)}"}
    W, H, n = s.width, s.height, s.width * s.height
    learned_spp = [1, 2, 4, 8, 16, 20, 24, 26, 28, 30, 32, 36, 40, 48, 64]
    flip_counts = [1, 2, 4]  # the learned result averaged over this many mirrored network passes
    plain_spp = [64, 128, 256, 512]
    tr = px.Tracer.of(gpu, s)
    tr.set_kernel(kernel)
    net = Unet.pretrained(gpu)
    frame = 0
    while frame < args.ref_spp:
        c = min(64, args.ref_spp - frame)
        tr.trace(cam, W, H, frame, c)
        frame += c
    prev = tr.image()
    ref = T.radiance(T.px_diff(prev, None, n), W, H)
    buf = px.GpuArray(gpu, (34 * n + 1) * 4)
    hbuf = px.GpuArray(gpu, n * 16)
    rel_plain, rel_learned, kept = {}, {}, {}
    tiles = ((W + TILE - 1) // TILE) * ((H + TILE - 1) // TILE)
    # relMSE of one frame swings by ~10 % between sample sets (a few bright
    # paths decide it): every figure is the mean over `relmse_frames`
    # independent frames
    for _ in range(args.relmse_frames):
        for spp in learned_spp + plain_spp:
            # traced in two halves: the first half's image is the learned
            # denoiser's part-way snapshot (the plain method ignores it)
            first = spp // 2
            mid = None
            if first > 0:
                tr.trace(cam, W, H, frame, first)
                mid = tr.image()
            tr.trace(cam, W, H, frame + first, spp - first)
            frame += spp
            img = tr.image()
            noisy = T.px_diff(img, prev, n)
            half = None if mid is None else snapshot_host(T.px_diff(mid, prev, n), W, H)
            prev = img
            buf.write(noisy)
            kernels.denoise(gpu, buf, W, H)
            rel_plain.setdefault(spp, []).append(T.relmse(T.radiance(buf.read(np.uint32), W, H), ref))
            if spp in learned_spp:
                if half is not None:
                    hbuf.write(half)
                for fl in flip_counts:
                    net.set_flips(fl)
                    buf.write(noisy)
                    kept.setdefault((fl, spp), []).append(
                        net.denoise_px(buf, W, H, half=hbuf if half is not None else None, tile=TILE,
                                       threshold=THRESHOLD, count=True) / tiles)
                    rel_learned.setdefault((fl, spp), []).append(
                        T.relmse(T.radiance(buf.read(np.uint32), W, H), ref))
    buf.free()
    rel_plain_frames = rel_plain
    rel_plain = {k: float(np.mean(v)) for k, v in rel_plain.items()}
    target = rel_plain[args.plain_spp]
    # the flip count with the fewest samples to reach the plain figure (ties: fewer passes)
    best_fl = min(flip_counts, key=lambda fl: (next((p for p in learned_spp
                                                      if np.mean(rel_learned[(fl, p)]) <= target), 1 << 30), fl))
    spread = {"plain": {str(k): [round(x, 6) for x in v] for k, v in rel_plain_frames.items() if k == args.plain_spp},
              "learned": {str(k): [round(x, 6) for x in rel_learned[(best_fl, k)]] for k in (24, 28, 32, 48)}}
    by_flips = {str(fl): {str(p): round(float(np.mean(rel_learned[(fl, p)])), 6) for p in learned_spp}
                for fl in flip_counts}
    kept = {p: float(np.mean(kept[(best_fl, p)])) for p in learned_spp}
    rel_learned = {p: float(np.mean(rel_learned[(best_fl, p)])) for p in learned_spp}
    net.set_flips(best_fl)

    def frame_ms(spp, learned, reps):
        def once():
            if learned and spp >= 2:
                tr.trace(cam, W, H, 0, spp // 2)
                tr.snapshot(hbuf)
                tr.trace(cam, W, H, spp // 2, spp - spp // 2)
                net.denoise(tr, half=hbuf)
            elif learned:
                tr.trace(cam, W, H, 0, spp)
                net.denoise(tr)
            else:
                tr.trace(cam, W, H, 0, spp)
                tr.denoise()
        once()
        gpu.wait(60000)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            once()
        b.record(stream)
        gpu.wait(60000)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    t_plain = frame_ms(args.plain_spp, False, 2)
    match = next((p for p in learned_spp if rel_learned[p] <= target), None)
    out = {
        "reference_spp": args.ref_spp,
        "frames": args.relmse_frames,
        "relmse_per_frame": spread,
        "plain": {"spp": args.plain_spp, "relmse": round(target, 6), "frame_ms": round(t_plain, 3),
                  "frames_per_s": round(1000.0 / t_plain, 3)},
        "relmse_plain_denoise": {str(k): round(v, 6) for k, v in rel_plain.items()},
        "relmse_learned": {str(k): round(v, 6) for k, v in rel_learned.items()},
        "flips": best_fl,
        "relmse_learned_by_flips": by_flips,
        "fallback_tile_share": {str(k): round(v, 4) for k, v in kept.items()},
        "threshold": THRESHOLD,
    }
    if match is not None:
        t_l = frame_ms(match, True, 3)
        out["learned"] = {"spp": match, "relmse": round(rel_learned[match], 6), "frame_ms": round(t_l, 3),
                          "frames_per_s": round(1000.0 / t_l, 3)}
        out["speedup_at_equal_relmse"] = round(t_plain / t_l, 2)
        # the spp where the learned curve crosses the target (log-log between the
        # measured neighbours), with the frame time scaled by samples: a
        # finer estimate than the measured grid point, reported beside it
        k = learned_spp.index(match)
        if k > 0:
            s0, s1 = learned_spp[k - 1], match
            r0, r1 = rel_learned[s0], rel_learned[s1]
            f = (np.log(target) - np.log(r0)) / (np.log(r1) - np.log(r0))
            s_eq = float(np.exp(np.log(s0) + f * (np.log(s1) - np.log(s0))))
            t_net = frame_ms(1, True, 3) - frame_ms(1, False, 3) + 0.0
            t_trace_1 = (frame_ms(match, False, 2) - frame_ms(1, False, 3)) / max(match - 1, 1)
            t_eq = frame_ms(1, False, 3) + t_trace_1 * (s_eq - 1) + t_net
            out["interpolated"] = {"spp": round(s_eq, 2), "frame_ms": round(t_eq, 3),
                                   "speedup": round(t_plain / t_eq, 2)}
    else:
        out["learned"] = None
        out["speedup_at_equal_relmse"] = None
    hbuf.free()
    net.close()
    tr.close()
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5"],
                    help="c2: the headline frame benchmark; c3: the skinned-animation stage timings; "
                         "c4: the learned denoiser's network alone; c5: batched serving")
    ap.add_argument("--scenes", type=int, default=64, help="scenes of the c5 workload")
    ap.add_argument("--frames", type=int, default=120, help="frames of the c3 workload")
    ap.add_argument("--ref-spp", type=int, default=4096, help="samples of the equal-relMSE reference render")
    ap.add_argument("--plain-spp", type=int, default=256, help="samples of the plain tracer + Denoise")
    ap.add_argument("--no-denoised", action="store_true", help="skip the equal-relMSE comparison")
    ap.add_argument("--relmse-frames", type=int, default=5,
                    help="independent frames each equal-relMSE figure is averaged over")
    ap.add_argument("--walk", type=int, default=0,
                    help="ray walk of --phase rays: 0 a thread per ray, 1 persistent, 2 sorted, 3 the 4-wide tree "
                         "(persistent), 4 the 4-wide tree (a thread per ray)")
    ap.add_argument("--adapt", default="",
                    help="--phase render with Adaptive Sampling: 'threshold,min samples,step' (off by default)")
    ap.add_argument("--stack", type=int, default=0,
                    help="stack placement of --phase rays thread-per-ray walks: 0 local, 1 shared, 2 registers")
    ap.add_argument("--tree", type=int, default=0, help="tree of --phase runs: 0 the LBVH, 1 the binned SAH tree")
    ap.add_argument("--kernel", type=int, default=-1,
                    help="render kernel id of --phase render (KERNEL_NAMES order; default: the tracer's default)")
    ap.add_argument("--phase", default="all", choices=["all", "render", "rays", "build", "nn"],
                    help="all: the benchmark; render/rays/build: only that kernel's launches (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload == "c3":
        run_c3(args)
        return
    if args.workload == "c4":
        run_c4(args)
        return
    if args.workload == "c5":
        run_c5(args)
        return

    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    import phiray_b200 as px
    from phiray_b200 import scenes

    s = scenes.c2_mesh(spp=args.spp)
    cam = px.camera(s)
    cam["w"], cam["h"] = s.width, s.height
    W, H, n = s.width, s.height, s.width * s.height
    gpu = px.Gpu(local)
    stream = torch.cuda.ExternalStream(gpu.stream)
    tr = px.Tracer.of(gpu, s)
    verts_dev = torch.tensor(s.verts, device=f"cuda:{local}")

    def step():
        tr.repose_device(verts_dev, rebuild=True)  # LBVH rebuild on the device
        tr.trace(cam, W, H, 0, args.spp)
        tr.denoise()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        gpu.wait(60000)
        torch.cuda.synchronize()

    if args.phase != "all":
        tr.set_tree(args.tree)
        profile_phase(args, tr, gpu, cam, verts_dev, W, H, n, local)
        gpu.close()
        return

    # The tree for this step: the SAH tree where its build costs less than
    # the trace time it saves over the step's samples (build + spp/4 frames
    # of 4 spp each), else the LBVH; then the render kernel on that tree.
    nf = s.ntris
    build_ms = timed_fn(gpu, stream, lambda: tr.repose_device(verts_dev, rebuild=True), 10)
    refit_ms = timed_fn(gpu, stream, lambda: tr.repose_device(verts_dev, rebuild=False), 10)
    tree, tree_ms = tr.autotune_tree(cam, W, H, 4, max(1, args.spp // 4))
    sah_build_ms = timed_fn(gpu, stream, lambda: tr.set_tree(px.Tracer.TREE_SAH), 3)
    tr.set_tree(tree)
    chosen, tune_ms = tr.autotune(cam, W, H, 4)  # the render kernel for this scene (keeps the image contract)
    launches = count_launches(step)
    for _ in range(args.warmup):
        step()
    barrier()
    _, rays_per_frame = tr.time()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        barrier()
    ms_step = max_over_ranks(e0.elapsed_time(e1) / args.steps, f"cuda:{local}")
    value = whole_job_rate(rays_per_frame, world, ms_step) / 1e6

    # End to end through the public API from pinned host memory.
    pin = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for k, a in
           (("v", s.verts), ("f", s.faces.view(np.int32)), ("m", s.mats))}
    hv, hf, hm = pin["v"].numpy(), pin["f"].numpy().view(np.uint32), pin["m"].numpy()
    h2d = hv.nbytes + hf.nbytes + hm.nbytes + cam.nbytes
    d2h = n * 4

    e2e_parts = {"create_ms": 0.0, "trace_denoise_ms": 0.0, "read_ms": 0.0, "close_ms": 0.0}

    def e2e_step():
        t0 = time.perf_counter()
        t = px.Tracer(gpu, hv, hf, hm)
        if tree != px.Tracer.TREE_LBVH:
            t.set_tree(tree)  # the tree the autotuner picked (rebuilt over the uploaded faces)
        t.set_kernel(chosen)  # the render kernel the autotuner picked for this scene
        gpu.wait(60000)
        t1 = time.perf_counter()
        t.trace(cam, W, H, 0, args.spp)
        t.denoise()
        gpu.wait(60000)
        t2 = time.perf_counter()
        img = t.pixels()
        t3 = time.perf_counter()
        t.close()
        t4 = time.perf_counter()
        for k, a, b in (("create_ms", t0, t1), ("trace_denoise_ms", t1, t2), ("read_ms", t2, t3), ("close_ms", t3, t4)):
            e2e_parts[k] += (b - a) * 1e3
        return img

    e2e_step()
    barrier()
    for k in e2e_parts:
        e2e_parts[k] = 0.0
    e2e_steps = max(7, args.steps)
    e2e_each = []
    with Clocks(local) as e2e_clk:
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ts = time.perf_counter()
            e2e_step()
            e2e_each.append((time.perf_counter() - ts) * 1e3)
        barrier()
        e2e_mean_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, f"cuda:{local}")
        # the median step: one step held up by something outside this process
        # (seen once at 906 ms against 219 ms, clocks steady) does not decide
        # the figure; the mean is printed beside it
        e2e_s = max_over_ranks(statistics.median(e2e_each) * 1e-3, f"cuda:{local}")
    e2e = whole_job_rate(rays_per_frame, world, e2e_s * 1e3) / 1e6
    e2e_mean = whole_job_rate(rays_per_frame, world, e2e_mean_s * 1e3) / 1e6

    # Phase timings (same device, outside the headline loop).
    def timed(fn, reps):
        return timed_fn(gpu, stream, fn, reps)

    tree_build_ms = timed(lambda: tr.repose_device(verts_dev, rebuild=True), 5)
    tr.trace(cam, W, H, 0, args.spp)
    trace_ms, trace_rays = tr.time()
    denoise_ms = timed(lambda: tr.denoise(), 5)
    counts = tr.trace_stats(cam, W, H, 0, args.spp)  # same walks, counted
    alg_bytes = counts[1] * 64 + counts[2] * 48
    pk = peaks()
    achieved = alg_bytes / (trace_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "trace_render_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tinfo = json.load(f)
        traffic = tinfo.get("dram_bytes_per_launch_full")

    rays = torch.empty((n, 8), dtype=torch.float32, device=f"cuda:{local}")
    hits = torch.empty((n, 4), dtype=torch.float32, device=f"cuda:{local}")
    tr.secondary_rays(cam, W, H, 0, rays)
    walk_ms = {}
    # (walk schedule, stack placement of the thread-per-ray walk)
    walks = {"thread_per_ray": (px.Tracer.WALK_THREAD, px.Tracer.STACK_LOCAL),
             "thread_per_ray_shared_stack": (px.Tracer.WALK_THREAD, px.Tracer.STACK_SHARED),
             "thread_per_ray_register_stack": (px.Tracer.WALK_THREAD, px.Tracer.STACK_REGISTER),
             "persistent_fetch": (px.Tracer.WALK_FETCH, px.Tracer.STACK_LOCAL),
             "sorted_fetch": (px.Tracer.WALK_SORTED, px.Tracer.STACK_LOCAL),
             "wide_fetch": (px.Tracer.WALK_WIDE, px.Tracer.STACK_LOCAL),
             "wide_thread_per_ray": (px.Tracer.WALK_WIDE_THREAD, px.Tracer.STACK_LOCAL)}
    tree_names = {px.Tracer.TREE_LBVH: "lbvh", px.Tracer.TREE_SAH: "sah"}
    for t_kind in (px.Tracer.TREE_LBVH, px.Tracer.TREE_SAH):
        tr.set_tree(t_kind)
        for name, (mode, place) in walks.items():
            tr.set_walk(mode)
            tr.set_stack(place)
            tr.trace_rays(rays, n, hits, False)  # (the wide walk collapses its tree here, untimed)
            walk_ms[f"{tree_names[t_kind]}/{name}"] = timed(lambda: tr.trace_rays(rays, n, hits, False), 10)
    best_walk = min(walk_ms, key=walk_ms.get)
    inc_ms = walk_ms[best_walk]
    tr.set_tree({"lbvh": px.Tracer.TREE_LBVH, "sah": px.Tracer.TREE_SAH}[best_walk.split("/")[0]])
    tr.set_walk(walks[best_walk.split("/")[1]][0])
    tr.set_stack(walks[best_walk.split("/")[1]][1])
    _, inc_steps, inc_tests = tr.trace_rays_stats(rays, n, hits, False)
    node_bytes = 128 if "/wide" in best_walk else 64
    inc_bytes = inc_steps * node_bytes + inc_tests * 48
    tr.set_walk(px.Tracer.WALK_THREAD)
    tr.set_stack(px.Tracer.STACK_LOCAL)
    tr.set_tree(tree)
    ids = torch.empty(n, dtype=torch.int32, device=f"cuda:{local}")
    ts = torch.empty(n, dtype=torch.float32, device=f"cuda:{local}")
    prim_ms = timed(lambda: tr.primary(cam, W, H, 0, ids, ts), 10)

    denoised = None if args.no_denoised else equal_relmse(args, gpu, s, cam, stream, chosen)

    out = None
    if rank == 0:
        cpu = None if args.no_cpu else cpu_baseline(s, cam)
        out = {
            "metric": METRIC,
            "value": round(value, 2),
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_step, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": dict(C2_CONFIG) if (W, H, args.spp, s.bounces, nf) == (1920, 1080, 64, 8, 1310722) else
            {"workload": WORKLOAD, "frame": f"{W}x{H}", "spp": args.spp, "bounces": s.bounces, "tris": nf},
            "parallelism": f"replicas x{world}",
            "l2": "scene ~300 MB of nodes/triangles/materials > 126 MB L2; the rebuild rewrites them each step",
            "render_kernel": {"chosen": KERNEL_NAMES[chosen],
                              "ms_4spp": {KERNEL_NAMES[k]: round(v, 3) for k, v in enumerate(tune_ms)}},
            "frames_per_s": round(1000.0 / ms_step * world, 3),
            "rays_per_frame": int(rays_per_frame),
            "tree": {"chosen": tree_names[tree],
                     "autotune_ms": dict(zip(("lbvh_build", "lbvh_trace_4spp", "sah_build", "sah_trace_4spp"),
                                             [round(v, 3) for v in tree_ms])),
                     "frames_weighed": max(1, args.spp // 4)},
            "phases_ms": {"lbvh_build": round(build_ms, 3), "lbvh_refit": round(refit_ms, 3),
                          "sah_build": round(sah_build_ms, 3), "tree_rebuild_in_step": round(tree_build_ms, 3),
                          "trace": round(trace_ms, 3), "denoise": round(denoise_ms, 3)},
            "lbvh_build_gbs": round(412 * nf / (build_ms * 1e-3) / 1e9, 1),
            "lbvh_refit_gbs": round(172 * nf / (refit_ms * 1e-3) / 1e9, 1),
            "incoherent_grays": round(n / (inc_ms * 1e-3) / 1e9, 3),
            "incoherent_grays_by_walk": {k: round(n / (v * 1e-3) / 1e9, 3) for k, v in walk_ms.items()},
            "incoherent_walk": {"best": best_walk, "node_bytes": node_bytes,
                                "steps_per_ray": round(inc_steps / n, 2), "tests_per_ray": round(inc_tests / n, 2),
                                "achieved_gbs": round(inc_bytes / (inc_ms * 1e-3) / 1e9, 1),
                                "frac_of_hbm": round(inc_bytes / (inc_ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4)},
            "primary_grays": round(n / (prim_ms * 1e-3) / 1e9, 3),
            "roofline": {"bound": "hbm", "kernel": "k_render (path-trace megakernel)", "achieved": round(achieved, 1),
                         "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / pk["hbm_gbs"], 4),
                         "traffic": traffic, "peak_source": pk["source"],
                         "algorithmic": f"{counts[1]} node steps x 64 B + {counts[2]} triangle tests x 48 B per launch"},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e, 2), "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "statistic": "median step", "mean_value": round(e2e_mean, 2),
                    "steps": e2e_steps, "step_ms": [round(v, 1) for v in e2e_each],
                    "phases_ms": {k: round(v / e2e_steps, 1) for k, v in e2e_parts.items()},
                    "clocks": e2e_clk.summary()},
            "denoised": denoised,
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(out), flush=True)
    gpu.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
