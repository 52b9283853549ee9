"""Benchmark: samples/s of the path-tracing hot path on one B200 (or N, weak scaling).

Workload (default): the metallic x roughness sphere grid — 7x7 UV spheres of
64x32 segments (200,706 triangles with the floor), a 512^2 sRGB checker floor
texture with trilinear mips, one directional and one point light, sky 0.3;
512x512 pixels, 256 samples per pixel, 8 bounces. One step = one frame:
`PathTracer.refine(256)` on the resident scene (67,108,864 camera paths).

Reported (one JSON line from rank 0):
  value      samples/s over all ranks, device time (CUDA events on the
             library's stream around the path-tracing kernels), max over ranks;
  e2e        the same metric through `PathTraceCudaRenderer.render` (scene
             upload with the host BVH build, refine, image readback), wall time;
  roofline   the path kernel's algorithmic bytes (per-ray / per-vertex byte
             model of the design notes, from device counters) / kernel time,
             against the measured HBM copy bandwidth;
  cpu_baseline  the CPU restatement of the reference (oracle) on this host's
             cores on a bounded sample of the same frame.
`--impl reference` times that CPU restatement alone (the Rust reference has no
toolchain here) on the same workload and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
import __graft_entry__ as entry  # noqa: E402

METRIC = "samples/s & Mrays/s vs plain GPU path; p50/p99 request latency at PSNR≥45dB"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
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

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(name: str):
    ts = entry.load_package().testscenes
    if name == "c1":
        scene, opts = ts.sphere_grid_c1(512, 256)
        return scene, opts, None, "sphere_grid_7x7_64x32 512x512 256spp 8 bounces (200,706 tris)"
    if name == "c0":
        scene, opts = ts.cornell_c0()
        return scene, opts, None, "cornell_unit_box 256x256 64spp 8 bounces (36 tris)"
    if name == "c2":
        scene, opts, env = ts.stress_c2()
        return scene, opts, env, "stress_heightfield_spheres 1920x1080 64spp 8 bounces (~4.1M tris, env 512x256)"
    if name == "soup":
        scene = ts.random_soup(500_000, seed=107)
        opts = ts.pt_opts(1024, 16, 8, h=768, scene_camera=0, ambient=0.1)
        return scene, opts, None, "random_soup 500k tris (mixed-workload scene class) 1024x768 16spp 8 bounces"
    raise SystemExit(f"unknown config {name}")


_MIXED_SCENES = {}


def mixed_scene(k: int, stress_grid: int = 1024, stress_spheres: int = 500):
    """Scene k of the mixed workload (built once): 0 Cornell box, 1 sphere
    grid, 2 stress scene, 3-10 random soups of 10k-500k triangles."""
    if k in _MIXED_SCENES:
        return _MIXED_SCENES[k]
    ts = entry.load_package().testscenes
    if k == 0:
        s, o = ts.cornell_c0()
        v = (s, o, None)
    elif k == 1:
        s, o = ts.sphere_grid_c1(512, 256)
        v = (s, o, None)
    elif k == 2:
        v = ts.stress_c2(grid=stress_grid, spheres=stress_spheres)
    else:
        tris = int(np.random.default_rng(100 + k).integers(10_000, 500_001))
        s = ts.random_soup(tris, seed=100 + k)
        v = (s, ts.pt_opts(64, 1, 8, scene_camera=0, ambient=0.1), None)
    _MIXED_SCENES[k] = v
    return v


def mixed_requests(n: int, seed: int):
    """The batched workload: `n` requests, each drawing its scene uniformly
    from {Cornell box, sphere grid, stress scene, 8 random soups of
    10k-500k triangles}, its resolution from {128^2, 256^2, 512^2, 1024x768},
    its spp from {1, 4, 16, 64} and its bounce limit from {2, 4, 8}."""
    from oxideav_render_b200.options import PathTraceOptions
    rng = np.random.default_rng(seed)
    res = [(128, 128), (256, 256), (512, 512), (1024, 768)]
    out = []
    for i in range(n):
        k = int(rng.integers(0, 11))
        w, h = res[int(rng.integers(0, 4))]
        spp = [1, 4, 16, 64][int(rng.integers(0, 4))]
        b = [2, 4, 8][int(rng.integers(0, 3))]
        s, o, env = mixed_scene(k)
        opts = o.replace(width=w, height=h, path_trace=PathTraceOptions(samples_per_pixel=spp, max_bounces=b,
                                                                        seed=i))
        out.append((k, s, opts, env))
    return out


def run_mixed(ctx, api, torch, n_requests: int, seed: int, check: int = 8):
    """Plain per-request GPU path (each request synced, refined and read back
    alone, one after another) against the batched path (all requests in one
    pt_tracer_refine_many call, then read back). Returns the comparison."""
    reqs = mixed_requests(n_requests, seed)
    tracers = []
    for k, s, o, env in reqs:
        t = api.PathTracer(ctx)
        if env is not None:
            t.set_environment(api.EnvironmentMap(env))
        t.sync(s, o)
        tracers.append(t)
    total = sum(o.width * o.height * o.path_trace.samples_per_pixel for _, _, o, _ in reqs)
    # Warm-up (loads modules, allocates wave buffers).
    api.refine_many(ctx, tracers[:4], [1] * 4)
    for t in tracers[:4]:
        t.reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for t, (_, _, o, _) in zip(tracers, reqs):
        t.refine(o.path_trace.samples_per_pixel)
        t.hdr()
    plain_s = time.perf_counter() - t0
    plain_acc = [tracers[i].accum() for i in range(min(check, len(tracers)))]
    for t in tracers:
        t.reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    api.refine_many(ctx, tracers, [o.path_trace.samples_per_pixel for _, _, o, _ in reqs])
    for t in tracers:
        t.hdr()
    batched_s = time.perf_counter() - t0
    st = api.batch_stats(ctx)
    identical = all(np.array_equal(tracers[i].accum(), plain_acc[i]) for i in range(len(plain_acc)))
    for t in tracers:
        t.close()
    return {"requests": n_requests, "samples": int(total), "plain_s": plain_s, "batched_s": batched_s,
            "plain_samples_per_s": total / plain_s, "batched_samples_per_s": total / batched_s,
            "speedup": plain_s / batched_s, "batched_waves": st["waves"],
            "batched_mrays_per_s": st["rays"] / (st["ms"] / 1000.0) / 1e6 if st["ms"] > 0 else None,
            "bit_identical_checked": len(plain_acc), "bit_identical": identical,
            "timing": "wall clock, host submit to HDR readback of every request"}


def serving_scenes(n: int, seed: int):
    """The served workload's resident scenes: the mixed workload's eleven
    (Cornell box, sphere grid, ~4.1M-triangle stress scene, eight soups)
    plus random soups of 10k-1M triangles (log-uniform) up to `n`."""
    ts = entry.load_package().testscenes
    out = [mixed_scene(k) for k in range(11)]
    rng = np.random.default_rng(seed + 1)
    for k in range(11, n):
        tris = int(np.exp(rng.uniform(np.log(10_000), np.log(1_000_000))))
        s = ts.random_soup(tris, seed=1000 + k)
        out.append((s, ts.pt_opts(64, 1, 8, scene_camera=0, ambient=0.1), None))
    return out


def run_served(ctx, api, torch, args):
    """Poisson arrivals of mixed requests against the render server, per
    arrival rate: p50/p99 latency (submit -> HDR in host memory) and the
    delivered samples/s; beside it the plain per-request path on a bounded
    sample of the same requests, timed back to back."""
    from oxideav_render_b200.options import PathTraceOptions
    from oxideav_render_b200.serve import RenderServer
    t0 = time.perf_counter()
    scenes = serving_scenes(args.serve_scenes, 2026)
    gen_s = time.perf_counter() - t0
    srv = RenderServer(ctx, hbm_budget_bytes=int(args.serve_budget_gb * (1 << 30)), autotune=args.autotune,
                       wave_overlap=args.wave_overlap, wave_slots=args.serve_wave_slots)
    t0 = time.perf_counter()
    keys = [srv.register(s, o, api.EnvironmentMap(e) if e is not None else None) for s, o, e in scenes]
    register_s = time.perf_counter() - t0
    # Make every scene resident (one tiny request each), as a warm server is.
    t0 = time.perf_counter()
    warm = [srv.submit(k, o.replace(width=16, height=16, path_trace=PathTraceOptions(samples_per_pixel=1)))
            for k, (_, o, _) in zip(keys, scenes)]
    for t in warm:
        srv.wait(t)
        srv.release(t)
    admit_s = time.perf_counter() - t0
    res = [(128, 128), (256, 256), (512, 512), (1024, 768)]
    runs = []
    sample_reqs = None
    for rate in args.serve_rates:
        rng = np.random.default_rng(int(rate * 1000) + 17)
        n = max(8, min(int(rate * args.serve_seconds), args.serve_max))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        spec = []
        for i in range(n):
            if i > 0 and rng.random() < 0.2:
                spec.append(("cont", int(rng.integers(0, i)), 16))
            else:
                k = int(rng.integers(0, len(scenes)))
                w, h = res[int(rng.integers(0, 4))]
                spp = [1, 4, 16, 64][int(rng.integers(0, 4))]
                b = [2, 4, 8][int(rng.integers(0, 3))]
                o = scenes[k][1].replace(width=w, height=h,
                                         path_trace=PathTraceOptions(samples_per_pixel=spp, max_bounces=b, seed=i))
                spec.append(("new", k, o))
        tickets, submit_t, samples = [None] * n, [0.0] * n, [0] * n
        start = time.perf_counter()
        for i, sp in enumerate(spec):
            delay = start + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            submit_t[i] = time.perf_counter()
            if sp[0] == "new":
                tickets[i] = srv.submit(keys[sp[1]], sp[2])
                samples[i] = sp[2].width * sp[2].height * sp[2].path_trace.samples_per_pixel
            else:
                base = sp[1]
                while spec[base][0] == "cont":
                    base = spec[base][1]
                o = spec[base][2]
                tickets[i] = srv.submit_continuation(tickets[sp[1]], sp[2])
                samples[i] = o.width * o.height * sp[2]
        lat, done_t, images = [], [], {}
        for i, t in enumerate(tickets):
            img, st = srv.wait(t)
            lat.append(st["latency_ms"])
            done_t.append(submit_t[i] + st["latency_ms"] / 1000.0)
            if spec[i][0] == "new" and len(images) < args.serve_check:
                images[i] = img
        makespan = max(done_t) - submit_t[0]
        stats = srv.stats()
        for t in tickets:
            srv.release(t)
        runs.append({"rate_per_s": rate, "requests": n, "continuations": sum(1 for s in spec if s[0] == "cont"),
                     "samples": int(sum(samples)), "makespan_s": makespan,
                     "samples_per_s": sum(samples) / makespan,
                     "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "max_ms": float(max(lat))})
        sample_reqs = (spec, arrivals, images)
    st = srv.stats()
    srv.close()

    # Plain per-request path on the saturated run's first --plain-requests new
    # requests (in arrival order; --plain-seconds caps the time): one-shot
    # render (scene prepared
    # and uploaded per request, PathTraceRenderer::render_hdr semantics),
    # once with this library's default preparation (device BVH for large
    # scenes) and once with the BVH built on the host as the reference's
    # TraceScene::new does; and refine + hdr on a tracer whose scene is
    # already uploaded.
    from oxideav_render_b200 import abi
    spec, arrivals, images = sample_reqs
    renderer = api.PathTraceCudaRenderer(ctx)
    plain_t, plain_n, resident_t, identical, arr = [], [], [], [], []
    host_t = []
    budget_end = time.perf_counter() + args.plain_seconds
    for i, sp in enumerate(spec):
        if sp[0] != "new":
            continue
        if len(plain_t) >= args.plain_requests or time.perf_counter() > budget_end:
            break
        s, _, e = scenes[sp[1]]
        o = sp[2]
        renderer.tracer_mut().set_environment(api.EnvironmentMap(e) if e is not None else None)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = renderer.render_hdr(s, o)
        plain_t.append(time.perf_counter() - t0)
        plain_n.append(o.width * o.height * o.path_trace.samples_per_pixel)
        arr.append(arrivals[i])
        if i in images:
            identical.append(bool(np.array_equal(img, images[i])))
        tr = renderer.tracer
        tr.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tr.refine(o.path_trace.samples_per_pixel)
        tr.hdr()
        resident_t.append(time.perf_counter() - t0)
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_HOST)
        try:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            renderer.render_hdr(s, o)
            host_t.append(time.perf_counter() - t0)
        finally:
            ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)
    renderer.tracer.close()
    # Latency of the plain path under the same arrivals: one request at a
    # time, first come first served (Lindley recursion on measured times).
    def fcfs_latency(times):
        free_at, lat = 0.0, []
        for a, s_ in zip(arr, times):
            begin = max(a, free_at)
            free_at = begin + s_
            lat.append(1000.0 * (free_at - a))
        return lat

    plain_lat, host_lat = fcfs_latency(plain_t), fcfs_latency(host_t)
    sat = max(runs, key=lambda r: r["rate_per_s"])
    plain_sps = sum(plain_n) / sum(plain_t)
    host_sps = sum(plain_n) / sum(host_t)
    resident_sps = sum(plain_n) / sum(resident_t)
    return {
        "scenes": len(scenes), "budget_gb": args.serve_budget_gb, "scene_gen_s": gen_s, "register_s": register_s,
        "first_admission_s": admit_s, "scene_uploads": st["scene_uploads"], "scene_evictions": st["scene_evictions"],
        "peak_resident_gb": st["peak_resident_bytes"] / (1 << 30), "waves": st["waves"],
        "gpu_mrays_per_s": st["rays"] / (st["gpu_ms"] / 1000.0) / 1e6 if st["gpu_ms"] > 0 else None,
        "runs": runs,
        "plain_render": {"requests": len(plain_t), "samples_per_s": plain_sps,
                         "p50_ms": float(np.percentile(plain_lat, 50)), "p99_ms": float(np.percentile(plain_lat, 99)),
                         "call": "PathTraceCudaRenderer.render_hdr per request (scene prepared + uploaded per call)"},
        "plain_render_host_bvh": {"requests": len(host_t), "samples_per_s": host_sps,
                                  "p50_ms": float(np.percentile(host_lat, 50)),
                                  "p99_ms": float(np.percentile(host_lat, 99)),
                                  "call": "the same one-shot render with the BVH built on the host per call"},
        "plain_resident": {"requests": len(resident_t), "samples_per_s": resident_sps,
                           "call": "PathTracer.refine + hdr per request, scene already on the device"},
        "speedup_vs_plain_render": sat["samples_per_s"] / plain_sps,
        "speedup_vs_plain_render_host_bvh": sat["samples_per_s"] / host_sps,
        "speedup_vs_plain_resident": sat["samples_per_s"] / resident_sps,
        "bit_identical_checked": len(identical), "bit_identical": all(identical) if identical else None,
    }


def algorithmic_bytes(ext_rays, shadow_rays, nodes, tris, samples):
    """Byte model per unit of work: per traced ray 32 B ray + 16 B hit, 64 B
    per BVH node visited, 48 B per triangle record tested; per shaded vertex
    16 B hit + 128 B path state read/write + 32 B per spawned ray; 32 B per
    accumulated sample (16 B read + 16 B write)."""
    rays = ext_rays + shadow_rays
    return (48 * rays + 64 * nodes + 48 * tris + ext_rays * (16 + 128) + 32 * (ext_rays + shadow_rays)
            + 32 * samples)


def profiled_traffic(kernel: str, config: str, wave_paths: int):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/<kernel>_*.md, line `traffic_bytes_per_launch | N`), scaled to
    this workload's launch size when the capture ran a smaller wave (line
    `profiled_wave_paths | M`): a launch's traffic grows with the paths it
    processes."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_*.md"))):
        text = open(path).read()
        m = re.search(r"traffic_bytes_per_launch \| (\d+)", text)
        if m and f"config={config}" in text:
            w = re.search(r"profiled_wave_paths \| (\d+)", text)
            scale = wave_paths / int(w.group(1)) if w else 1.0
            return int(int(m.group(1)) * scale)
    return None


def cpu_baseline(scene, opts, env, budget_s: float):
    """Oracle on this host's cores over a bounded band of rows of the frame."""
    orc = entry.load_oracle()
    from oxideav_render_b200.scene import Camera
    desc = scene.to_desc(opts)
    sc = orc.OracleScene(desc)
    cam = Camera.resolve(scene, opts, opts.width, opts.height)
    oenv = orc.OracleEnv(env) if env is not None else None
    cores = os.cpu_count() or 1
    # Rows spread evenly over the frame; calibrate at 1 spp, then size the
    # sample so it takes about `budget_s`.
    rows = min(64, opts.height)
    stride = max(opts.height // rows, 1)
    t0 = time.perf_counter()
    orc.refine_rows(sc, cam, opts, oenv, stride // 2, stride, rows, 0, 1, cores)
    dt = max(time.perf_counter() - t0, 1e-3)
    spp = max(1, min(opts.path_trace.samples_per_pixel, int(budget_s / dt)))
    t0 = time.perf_counter()
    _, rc = orc.refine_rows(sc, cam, opts, oenv, stride // 2, stride, rows, 0, spp, cores)
    dt = time.perf_counter() - t0
    n = opts.width * rows * spp
    return {"value": n / dt, "unit": "samples/s", "cores": cores, "kind": "port",
            "sample": f"every {stride}th row ({rows} of {opts.height}) x {spp} spp of the frame "
                      f"({n} camera paths, {dt:.1f} s)",
            "mrays_per_s": (rc[0] + rc[1]) / dt / 1e6}


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    from oxideav_render_b200 import shard
    return shard.max_over_ranks(x, device="cuda")


def barrier(ws: int):
    import torch
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        torch.cuda.synchronize()


def run_reference(args):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    pkg = entry.load_package()
    scene, opts, env, wname = workload(args.config)
    orc = entry.load_oracle()
    from oxideav_render_b200.scene import Camera
    desc = scene.to_desc(opts)
    sc = orc.OracleScene(desc)
    cam = Camera.resolve(scene, opts, opts.width, opts.height)
    oenv = orc.OracleEnv(env) if env is not None else None
    cores = os.cpu_count() or 1
    rows, spp = min(args.ref_rows, opts.height), args.ref_spp
    stride = max(opts.height // rows, 1)
    times, rays = [], 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _, rc = orc.refine_rows(sc, cam, opts, oenv, stride // 2, stride, rows, i * spp, spp, cores)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            rays += rc[0] + rc[1]
    n = opts.width * rows * spp
    value = n * len(times) / sum(times)
    sample = f"every {stride}th row ({rows} of {opts.height}) x {spp} spp per step ({n} camera paths)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": wname, "parallelism": "host threads"},
        "mrays_per_s": rays / sum(times) / 1e6,
        "cpu_baseline": {"value": value, "unit": "samples/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_raycast(ctx, api, torch, scene, opts, cpu: bool, steps: int = 3, pbr: bool = False):
    """RenderBackend::Raycast on the workload's scene and camera — Phong /
    Whitted (the default shading mode), or Pbr with ray-traced shadows:
    one-shot renders through RaycastCudaRenderer (scene prepared + uploaded
    per call, as the reference's render does) and raycasts of an
    already-uploaded scene, plus the oracle's CPU restatement of the same
    frame."""
    import ctypes as C
    from oxideav_render_b200.options import ShadingMode
    from oxideav_render_b200.scene import Camera
    o = opts.replace(shading=ShadingMode.Pbr, aa=1, shadows=True) if pbr else \
        opts.replace(shading=ShadingMode.Phong, aa=1)
    samples = o.width * o.height * o.aa * o.aa
    r = api.RaycastCudaRenderer(ctx)
    img = r.render(scene, o)
    one_shot = []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = r.render(scene, o)
        one_shot.append(time.perf_counter() - t0)
    cam = Camera.resolve(scene, o, o.width * o.aa, o.height * o.aa)
    desc = scene.to_desc(o)
    sid = ctx.upload(desc)
    c, ro = cam.to_c(), o.to_raycast_c(cam.near, cam.far)
    out = np.zeros((o.height, o.width, 4), np.uint8)
    resident = []
    for i in range(steps + 1):
        t0 = time.perf_counter()
        ctx.check(ctx.lib.pt_raycast_render(ctx.ptr, sid, C.byref(c), C.byref(ro), None, 0,
                                            out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size))
        if i > 0:
            resident.append(time.perf_counter() - t0)
    ctx.release(sid)
    what = (f"Pbr (glTF direct light with shadow rays, mirror / refraction / BLEND rays, depth {o.max_ray_depth}, "
            f"reflection cut-off {o.reflection_roughness_cutoff})" if pbr else
            f"Phong (Whitted: shadow, mirror and refraction rays, depth {o.max_ray_depth})")
    res = {"workload": f"{what} {o.width}x{o.height}, aa {o.aa}",
           "samples_per_frame": samples,
           "one_shot_ms": 1000 * statistics.median(one_shot),
           "one_shot_samples_per_s": samples / statistics.median(one_shot),
           "resident_ms": 1000 * statistics.median(resident),
           "resident_samples_per_s": samples / statistics.median(resident),
           "identical_to_oracle": None, "cpu_ms": None}
    if cpu:
        oracle = entry.load_oracle()
        t0 = time.perf_counter()
        _, want = oracle.raycast(scene, o)
        res["cpu_ms"] = 1000 * (time.perf_counter() - t0)
        res["cpu_threads"] = min(64, os.cpu_count() or 1)
        res["identical_to_oracle"] = bool(np.array_equal(img, want))
        if not res["identical_to_oracle"]:
            res["max_byte_difference"] = int(np.max(np.abs(img.astype(int) - want.astype(int))))
    return res


def run_uploads(args):
    """Profiling case: uploads the workload's scene `--upload-only` times
    (device BVH build and device mip chains) and prints the phase times."""
    import torch
    entry.load_package()
    from oxideav_render_b200 import abi, api
    scene, opts, env, wname = workload(args.config)
    ctx = api.Context(torch.cuda.current_device())
    ctx.set_bvh_builder(abi.PT_BVH_BUILD_DEVICE)
    desc = scene.to_desc(opts)
    runs = []
    for _ in range(args.upload_only):
        sid = ctx.upload(desc)
        runs.append({k: 1000 * v for k, v in ctx.upload_seconds(sid).items()})
        runs[-1]["bvh"] = ctx.bvh_stats(sid)
        ctx.release(sid)
    print(json.dumps({"workload": wname, "uploads_ms": runs}))
    ctx.close()


def run_raycasts(args):
    """Profiling case: `--raycast-only` frames of the workload's scene on the
    raycast backend, Phong then Pbr, on a resident scene, and the timings."""
    import torch
    entry.load_package()
    from oxideav_render_b200 import api
    scene, opts, env, wname = workload(args.config)
    ctx = api.Context(torch.cuda.current_device())
    out = {"workload": wname,
           "phong": run_raycast(ctx, api, torch, scene, opts, cpu=False, steps=args.raycast_only),
           "pbr": run_raycast(ctx, api, torch, scene, opts, cpu=False, steps=args.raycast_only, pbr=True)}
    print(json.dumps(out))
    ctx.close()


def run_b200(args):
    import torch
    ws, rank, local = dist_setup()
    pkg = entry.load_package()
    from oxideav_render_b200 import api
    scene, opts, env, wname = workload(args.config)
    if args.spp:
        opts = opts.replace(path_trace=opts.path_trace.__class__(**{**opts.path_trace.__dict__,
                                                                   "samples_per_pixel": args.spp}))
        wname += f" (override: {args.spp} spp)"
    spp = opts.path_trace.samples_per_pixel
    samples_per_step = opts.width * opts.height * spp
    ctx = api.Context(local if ws > 1 else torch.cuda.current_device())
    if not args.wave_overlap:
        ctx.set_wave_overlap(False)
    elif args.wave_arenas:
        ctx.set_wave_overlap(args.wave_arenas)
    if args.wave_slots:
        ctx.set_wave_slots(args.wave_slots)
    ctx.set_schedule({"megakernel": 0, "wavefront": 1}[args.schedule])
    if args.seed_per_rank and ws > 1:
        opts = opts.replace(path_trace=opts.path_trace.__class__(**{**opts.path_trace.__dict__, "seed": rank}))
    tracer = api.PathTracer(ctx)
    if env is not None:
        tracer.set_environment(api.EnvironmentMap(env))
    tracer.sync(scene, opts)
    tuned = None
    if args.autotune:
        # pt_autotune: calibration refines on a scratch accumulator pick this
        # scene class's configuration (images are identical under every one).
        t0 = time.perf_counter()
        tuned = ctx.autotune(tracer, 0)
        tuned["seconds"] = time.perf_counter() - t0
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    for _ in range(args.warmup):
        tracer.refine(spp)
    barrier(ws)
    kernel_ms, wall_ms = [], []
    ext = shadow = 0
    split = {"ext_nodes": 0, "ext_tris": 0, "sh_nodes": 0, "sh_tris": 0}
    stage = {k: 0.0 for k in api.PathTracer.STAGES}
    with ClockSampler(local if ws > 1 else torch.cuda.current_device()) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tracer.refine(spp)
            wall_ms.append(1000 * (time.perf_counter() - t0))
            kernel_ms.append(tracer.last_kernel_ms())
            e, s = tracer.ray_counts()
            ext, shadow = ext + e, shadow + s
            for k, v in tracer.traversal_split().items():
                split[k] += v
    barrier(ws)
    # Stage split: one more (untimed) frame with CUDA events between the
    # stages. Events need direct launches; the timed frames replay each wave
    # as one CUDA graph.
    ctx.set_stage_timing(True)
    flush.zero_()
    torch.cuda.synchronize()
    tracer.refine(spp)
    stage = {k: v * args.steps for k, v in tracer.stage_ms().items()}
    stage_frame_ms = tracer.last_kernel_ms()
    ctx.set_stage_timing(False)
    dev_s = max_over_ranks(sum(kernel_ms) / 1000.0, ws)
    value = samples_per_step * args.steps * ws / dev_s
    ms_per_step = 1000 * dev_s / args.steps
    rays = ext + shadow
    mrays = max(rays / (sum(kernel_ms) / 1000.0) / 1e6, 0.0)
    # Roofline of the dominant kernel: its algorithmic bytes / its device time.
    peak, peak_kind = load_peaks()
    n_samples = samples_per_step * args.steps
    stage_bytes = {
        "extend": 48 * ext + 64 * split["ext_nodes"] + 48 * split["ext_tris"],
        "shadow": 48 * shadow + 64 * split["sh_nodes"] + 48 * split["sh_tris"],
        "shade": ext * (16 + 128 + 32) + 32 * shadow,
        "megakernel": algorithmic_bytes(ext, shadow, split["ext_nodes"] + split["sh_nodes"],
                                        split["ext_tris"] + split["sh_tris"], 0),
        "accumulate": 32 * n_samples,
    }
    dom = max((k for k in stage_bytes if stage[k] > 0), key=lambda k: stage[k])
    achieved = stage_bytes[dom] / (stage[dom] / 1000.0) / 1e9
    kernel_names = {"extend": "k_wf_extend", "shade": "k_wf_shade", "shadow": "k_wf_shadow",
                    "megakernel": "k_megakernel", "accumulate": "k_accumulate"}
    # Waves of the refine: the tuned wave size, else the one set or the
    # library's default (8,388,608 path slots).
    wave_slots = (tuned or {}).get("wave_slots") or args.wave_slots or (1 << 23)
    waves = max(math.ceil(samples_per_step / wave_slots), 1)
    iters = opts.path_trace.max_bounces + 1
    per_wave = (2 + 3 * iters) if args.schedule == "wavefront" else 2
    launches = args.steps * waves * per_wave
    launches_of_dom = args.steps * waves * (iters if args.schedule == "wavefront" and dom in
                                            ("extend", "shade", "shadow") else 1)
    traffic = profiled_traffic(kernel_names[dom], args.config, min(wave_slots, samples_per_step))

    # End to end: the reference-facing one-shot call (re-prepare + render + image).
    renderer = api.PathTraceCudaRenderer(ctx)
    if env is not None:
        renderer.tracer_mut().set_environment(api.EnvironmentMap(env))
    e2e_s, e2e_calls = [], []
    h2d = d2h = 0
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = renderer.render(scene, opts)
        dt = time.perf_counter() - t0
        e2e_calls.append({"wall_ms": 1000 * dt, "refine_device_ms": renderer.tracer.last_kernel_ms()})
        if i > 0:
            e2e_s.append(dt)
        h2d = ctx.scene_bytes(renderer.tracer.scene_id)
        d2h = img.nbytes
    e2e = None
    if e2e_s:
        e2e_t = max_over_ranks(sum(e2e_s) / len(e2e_s), ws)
        e2e = {"value": samples_per_step * ws / e2e_t, "unit": "samples/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": 1000 * e2e_t,
               "call": "PathTraceCudaRenderer.render (scene preparation and upload incl. the BVH build, "
                       "refine, sRGB image readback)",
               "calls": e2e_calls}
        # Where the host part of that time goes (one extra, separately timed upload).
        t0 = time.perf_counter()
        desc = scene.to_desc(opts)
        t1 = time.perf_counter()
        sid = ctx.upload(desc)
        t2 = time.perf_counter()
        e2e["host_ms"] = {"flatten": 1000 * (t1 - t0), "prepare_and_upload": 1000 * (t2 - t1),
                          "bvh_build": 1000 * ctx.bvh_stats(sid)["build_seconds"],
                          "bvh_on_device": ctx.bvh_on_device(sid),
                          "upload_phases": {k: 1000 * v for k, v in ctx.upload_seconds(sid).items()}}
        ctx.release(sid)
    raycast = raycast_pbr = None
    if args.raycast:
        raycast = run_raycast(ctx, api, torch, scene, opts, cpu=rank == 0 and not args.no_cpu_baseline)
        raycast_pbr = run_raycast(ctx, api, torch, scene, opts, cpu=rank == 0 and not args.no_cpu_baseline,
                                  pbr=True)
    mixed = None
    if args.mixed > 0:
        mixed = run_mixed(ctx, api, torch, args.mixed, 2026 + rank)
    served = None
    if args.serve_rates:
        served = run_served(ctx, api, torch, args)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(scene, opts, env, args.cpu_seconds)
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wname, "samples_per_step": samples_per_step, "global_batch": samples_per_step * ws,
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "flushed (256 MB write) before every timed step", "schedule": args.schedule,
                       "autotuned": tuned},
            "mrays_per_s": mrays, "rays_per_step": rays / args.steps, "wall_ms_per_step": statistics.mean(wall_ms),
            "stage_ms_per_step": {k: v / args.steps for k, v in stage.items() if v > 0},
            "stage_frame_ms": stage_frame_ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": kernel_names[dom],
                         "bytes_per_launch": stage_bytes[dom] / max(launches_of_dom, 1),
                         "ms_per_launch": stage[dom] / max(launches_of_dom, 1)},
            "e2e": e2e,
            "batched_mixed": mixed,
            "raycast": raycast,
            "raycast_pbr": raycast_pbr,
            "served": served,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(out))
    tracer.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "soup"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed-per-rank", action="store_true")
    ap.add_argument("--ref-rows", type=int, default=32)
    ap.add_argument("--ref-spp", type=int, default=8)
    ap.add_argument("--spp", type=int, default=0, help="override samples per pixel (profiling cases)")
    ap.add_argument("--schedule", default="wavefront", choices=["megakernel", "wavefront"])
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default configuration instead of pt_autotune's per-class choice")
    ap.add_argument("--mixed", type=int, default=64, help="requests in the batched-vs-plain comparison (0: skip)")
    ap.add_argument("--serve-rates", default="5,20,200",
                    help="Poisson arrival rates (requests/s) of the served runs, comma-separated ('' : skip)")
    ap.add_argument("--serve-seconds", type=float, default=8.0, help="arrival window per served run")
    ap.add_argument("--serve-max", type=int, default=96, help="requests per served run at most")
    ap.add_argument("--serve-scenes", type=int, default=32, help="resident scenes of the served runs")
    ap.add_argument("--serve-budget-gb", type=float, default=60.0, help="HBM budget of the resident scenes")
    ap.add_argument("--serve-check", type=int, default=8, help="served images compared with the plain path")
    ap.add_argument("--serve-wave-slots", type=int, default=0, help="path slots per served wave (0: the server's default)")
    ap.add_argument("--plain-requests", type=int, default=24, help="requests in the plain-path sample")
    ap.add_argument("--plain-seconds", type=float, default=60.0, help="time cap of the plain-path sample")
    ap.add_argument("--no-raycast", dest="raycast", action="store_false",
                    help="skip the RenderBackend::Raycast measurement")
    ap.add_argument("--upload-only", type=int, default=0,
                    help="profiling case: upload the scene this many times (device BVH, device mips) and exit")
    ap.add_argument("--no-wave-overlap", dest="wave_overlap", action="store_false",
                    help="trace one wave at a time instead of overlapping consecutive waves")
    ap.add_argument("--wave-slots", type=int, default=0,
                    help="path slots per wave (0: the library's default; autotune may override)")
    ap.add_argument("--wave-arenas", type=int, default=0,
                    help="waves in flight at once (2 or 3; 0: the library's default)")
    ap.add_argument("--raycast-only", type=int, default=0,
                    help="profiling case: this many raycast frames (Phong, then Pbr) of the scene and exit")
    args = ap.parse_args()
    args.serve_rates = [float(x) for x in args.serve_rates.split(",") if x.strip()]
    if args.warmup < 3:
        args.warmup = 3
    if args.upload_only > 0:
        run_uploads(args)
    elif args.raycast_only > 0:
        run_raycasts(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
