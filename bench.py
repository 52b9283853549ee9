"""Benchmark of the path-tracing hot path on one B200 (or N, weak scaling):
the served / batched form against the plain per-request GPU path.

Headline workload (config 3): a mix of 64 render requests, each drawing its
scene uniformly from {Cornell box C0, sphere grid C1, the ~4.1M-triangle
stress scene C2 with environment map and emitters, 8 random soups of
10k-500k triangles}, its resolution from {128^2, 256^2, 512^2, 1024x768},
its spp from {1, 4, 16, 64} and its bounce limit from {2, 4, 8}. One step =
every request's samples (about 310 M camera paths).

Reported (one JSON line from rank 0):
  value       samples/s of the batched form: pt_tracer_refine_many over one
              tracer per request, scenes resident, device time of the waves
              (CUDA events on the library's stream), max over ranks;
  e2e         the same requests through the serving C ABI (pt_server_submit
              / pt_server_wait on a warm server), host request descriptors in,
              HDR images back to host memory, wall clock;
  vs_plain    the plain per-request GPU path on the SAME requests:
              PathTraceCudaRenderer.render_hdr per request (scene prepared and
              uploaded per call) and refine + hdr on an uploaded scene, with
              p50 / p99 latencies and the speed-ups;
  served_poisson  config 4: Poisson arrivals (5 and 200 requests/s over a 60 s
              window, 20 % +16 spp continuations) against 32 resident scenes
              under a 60 GB budget; p50 / p99 latency, samples/s, and the plain
              path on the same requests replayed under the same arrivals;
  roofline    the dominant kernel's algorithmic bytes (byte model from device
              counters) / its device time, against the measured HBM bandwidth;
  plain_frame the single C1 frame (512^2, 256 spp) as a secondary figure;
  cpu_baseline  the oracle (CPU restatement of the reference) on this host's
              cores over one row of every request of the mix.
`--impl reference` times that CPU restatement alone on the same request mix.
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


def mixed_requests(n: int, seed: int, seed_base: int = 0):
    """The batched workload: `n` requests, each drawing its scene uniformly
    from {Cornell box, sphere grid, stress scene, 8 random soups of
    10k-500k triangles}, its resolution from {128^2, 256^2, 512^2, 1024x768},
    its spp from {1, 4, 16, 64} and its bounce limit from {2, 4, 8}.
    Request i renders with sample seed `seed_base + i`."""
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
                                                                        seed=seed_base + i))
        out.append((k, s, opts, env))
    return out


def request_samples(o) -> int:
    return o.width * o.height * o.path_trace.samples_per_pixel


def percentiles(lat_ms):
    return {"p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
            "max_ms": float(np.max(lat_ms))}


def upload_resident(ctx, api, reqs, spatial: bool):
    """Uploads each distinct scene of the request mix once, as resident
    scenes: with the spatial-split tree (PT_BVH_BUILD_HOST_SPATIAL) when
    `spatial`, since a resident scene amortises the slower build."""
    from oxideav_render_b200 import abi
    ids, descs = {}, []
    ctx.set_bvh_builder(abi.PT_BVH_BUILD_HOST_SPATIAL if spatial else abi.PT_BVH_BUILD_AUTO)
    try:
        for k, s, o, _ in reqs:
            if k not in ids:
                d = s.to_desc(o)
                descs.append(d)
                ids[k] = ctx.upload(d)
    finally:
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)
    return ids, descs


def run_batched(ctx, api, torch, reqs, args, ws, flush):
    """Headline: the request mix refined in shared waves (pt_tracer_refine_many
    over one tracer per request, each scene uploaded once and resident).
    One step = every request's samples; device time of the waves (CUDA
    events on the library's stream)."""
    t0 = time.perf_counter()
    scene_ids, descs = upload_resident(ctx, api, reqs, args.spatial_bvh)
    upload_s = time.perf_counter() - t0
    tracers = []
    for k, s, o, env in reqs:
        t = api.PathTracer(ctx)
        if env is not None:
            t.set_environment(api.EnvironmentMap(env))
        t.sync_resident(scene_ids[k], s, o)
        tracers.append(t)
    spp = [o.path_trace.samples_per_pixel for _, _, o, _ in reqs]
    total = sum(request_samples(o) for _, _, o, _ in reqs)

    def step():
        for t in tracers:
            t.reset()
        flush.zero_()
        torch.cuda.synchronize()
        api.refine_many(ctx, tracers, spp)

    for _ in range(args.warmup):
        step()
    barrier(ws)
    ms, rays, waves = [], 0, 0
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for _ in range(args.steps):
            step()
            st = api.batch_stats(ctx)
            ms.append(st["ms"])
            rays += st["rays"]
            waves += st["waves"]
    barrier(ws)
    # One more (untimed) batch with CUDA events between the stages: the
    # stage split and the counters the roofline uses. Stage events need
    # direct launches on one stream, so this batch runs without overlap.
    ctx.set_stage_timing(True)
    step()
    bc = api.batch_counters(ctx)
    stage_batch_ms = api.batch_stats(ctx)["ms"]
    ctx.set_stage_timing(False)
    return tracers, {"ms": ms, "rays": rays, "waves": waves, "total": total, "counters": bc,
                     "stage_batch_ms": stage_batch_ms, "clocks": clocks.summary(), "scene_ids": scene_ids,
                     "descs": descs, "scene_upload_s": upload_s}


def register_scenes(srv, api, scenes):
    """Registers (scene, opts, env) triples and makes each resident with one
    tiny request, as a warm server holds them. Returns the keys."""
    from oxideav_render_b200.options import PathTraceOptions
    keys = [srv.register(s, o, api.EnvironmentMap(e) if e is not None else None) for s, o, e in scenes]
    warm = [srv.submit(k, o.replace(width=16, height=16, path_trace=PathTraceOptions(samples_per_pixel=1)))
            for k, (_, o, _) in zip(keys, scenes)]
    for t in warm:
        srv.wait(t)
        srv.release(t)
    return keys


def run_served_batch(ctx, api, torch, reqs, args, tracers):
    """End to end through the serving C ABI: the same requests submitted to a
    warm RenderServer (their 11 scenes resident) all at once, each HDR image
    copied back to host memory; wall time from the first submit to the last
    image. Request descriptors go host -> device, HDR images device -> host."""
    import ctypes as C
    from oxideav_render_b200 import abi
    from oxideav_render_b200.serve import RenderServer
    srv = RenderServer(ctx, wave_overlap=args.wave_overlap, wave_slots=args.serve_wave_slots,
                       spatial_bvh=args.spatial_bvh, pipeline_depth=args.serve_depth)
    try:
        kinds = sorted({k for k, _, _, _ in reqs})
        scenes = [mixed_scene(k) for k in kinds]
        keys = dict(zip(kinds, register_scenes(srv, api, scenes)))
        total = sum(request_samples(o) for _, _, o, _ in reqs)
        h2d = len(reqs) * C.sizeof(abi.pt_server_request)
        d2h = sum(o.width * o.height * 16 for _, _, o, _ in reqs)
        runs, identical = [], []
        for rep in range(args.e2e_steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tickets = [srv.submit(keys[k], o) for k, _, o, _ in reqs]
            lat = []
            for i, t in enumerate(tickets):
                img, st = srv.wait(t)
                lat.append(st["latency_ms"])
                if rep == 0 and i < args.serve_check:
                    identical.append(bool(np.array_equal(img, tracers[i].hdr())))
                srv.release(t)
            wall = time.perf_counter() - t0
            if rep > 0:  # the first pass is a warm-up
                runs.append({"wall_s": wall, **percentiles(lat)})
        st = srv.stats()
    finally:
        srv.close()
    wall = statistics.median(r["wall_s"] for r in runs)
    return {"value": total / wall, "walls_s": [r["wall_s"] for r in runs], "wall_stat": "median", "unit": "samples/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": 1000 * wall, "p50_ms": statistics.median(r["p50_ms"] for r in runs),
            "p99_ms": statistics.median(r["p99_ms"] for r in runs),
            "call": "pt_server_submit of every request at once to a warm server (scenes resident), "
                    "pt_server_wait copies each HDR image to host memory; wall clock first submit -> last image",
            "steps": len(runs), "server_gpu_mrays_per_s": st["rays"] / (st["gpu_ms"] / 1000.0) / 1e6
            if st["gpu_ms"] > 0 else None,
            "bit_identical_checked": len(identical), "bit_identical": all(identical) if identical else None}


def run_plain_requests(ctx, api, torch, reqs, tracers, passes: int = 3):
    """The plain per-request GPU path on the same requests, one after
    another in request order: PathTraceCudaRenderer.render_hdr per request
    (PathTraceRenderer::render_hdr: the scene prepared and uploaded per call,
    refine, HDR read back), and refine + hdr on the request's tracer whose
    scene is already uploaded. Each request's times are the median of
    `passes` passes (host-side preparation is sensitive to other load on the
    host). Latencies assume every request arrived at once (first come, first
    served)."""
    renderer = api.PathTraceCudaRenderer(ctx)
    one = [[] for _ in reqs]
    res = [[] for _ in reqs]
    for _ in range(passes):
        for i, ((k, s, o, env), t) in enumerate(zip(reqs, tracers)):
            renderer.tracer_mut().set_environment(api.EnvironmentMap(env) if env is not None else None)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            renderer.render_hdr(s, o)
            one[i].append(time.perf_counter() - t0)
            t.reset()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            t.refine(o.path_trace.samples_per_pixel)
            t.hdr()
            res[i].append(time.perf_counter() - t0)
    renderer.tracer.close()
    one = [statistics.median(x) for x in one]
    res = [statistics.median(x) for x in res]
    total = sum(request_samples(o) for _, _, o, _ in reqs)
    return {"one_shot": {"samples_per_s": total / sum(one), "wall_s": sum(one),
                         **percentiles(1000 * np.cumsum(one)),
                         "call": "PathTraceCudaRenderer.render_hdr per request (scene prepared + uploaded per call)"},
            "resident": {"samples_per_s": total / sum(res), "wall_s": sum(res),
                         **percentiles(1000 * np.cumsum(res)),
                         "call": "PathTracer.refine + hdr per request, its scene already on the device"},
            "passes": passes, "per_request_stat": "median"}


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


def served_spec(n: int, scenes, seed: int):
    """Config 4's requests: drawn like the batched mix over the resident
    scenes; 20 % are +16 spp continuations of an earlier request."""
    from oxideav_render_b200.options import PathTraceOptions
    rng = np.random.default_rng(seed)
    res = [(128, 128), (256, 256), (512, 512), (1024, 768)]
    spec = []
    for i in range(n):
        if i > 0 and rng.random() < 0.2:
            j = int(rng.integers(0, i))
            while spec[j][0] == "cont":
                j = spec[j][1]
            spec.append(("cont", j, 16))
        else:
            k = int(rng.integers(0, len(scenes)))
            w, h = res[int(rng.integers(0, 4))]
            spp = [1, 4, 16, 64][int(rng.integers(0, 4))]
            b = [2, 4, 8][int(rng.integers(0, 3))]
            o = scenes[k][1].replace(width=w, height=h,
                                     path_trace=PathTraceOptions(samples_per_pixel=spp, max_bounces=b, seed=i))
            spec.append(("new", k, o))
    samples = []
    for sp in spec:
        o = sp[2] if sp[0] == "new" else spec[sp[1]][2]
        samples.append(o.width * o.height * (o.path_trace.samples_per_pixel if sp[0] == "new" else sp[2]))
    return spec, samples


def run_poisson(ctx, api, torch, args):
    """Config 4: Poisson arrivals of `served_spec` requests against a warm
    server holding 32 scenes under the HBM budget, per arrival rate (the
    requests of a rate arrive over --serve-seconds, at most --serve-max);
    p50/p99 latency (submit -> HDR in host memory) and delivered samples/s.
    The plain per-request path runs the SAME requests, continuations
    included: a new request is one PathTraceCudaRenderer.render_hdr (scene
    prepared + uploaded), a continuation refine(16) + hdr on its base
    request's renderer (PathTracer::refine on a live tracer). Its latencies
    under each rate's arrivals follow from the measured service times, one
    request at a time in arrival order (Lindley's recursion)."""
    from oxideav_render_b200.serve import RenderServer
    t0 = time.perf_counter()
    scenes = serving_scenes(args.serve_scenes, 2026)
    gen_s = time.perf_counter() - t0
    n = max(8, min(int(max(args.serve_rates) * args.serve_seconds), args.serve_max))
    spec, samples = served_spec(n, scenes, 4242)
    srv = RenderServer(ctx, hbm_budget_bytes=int(args.serve_budget_gb * (1 << 30)), wave_overlap=args.wave_overlap,
                       wave_slots=args.serve_wave_slots, spatial_bvh=args.spatial_bvh, pipeline_depth=args.serve_depth)
    t0 = time.perf_counter()
    keys = register_scenes(srv, api, scenes)
    register_s = time.perf_counter() - t0
    runs, images = [], {}
    for rate in args.serve_rates:
        m = max(8, min(int(rate * args.serve_seconds), n))
        arrivals = np.cumsum(np.random.default_rng(int(rate * 1000) + 17).exponential(1.0 / rate, m))
        tickets, lat = [None] * m, [0.0] * m
        start = time.perf_counter()
        for i in range(m):
            delay = start + arrivals[i] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            sp = spec[i]
            tickets[i] = (srv.submit(keys[sp[1]], sp[2]) if sp[0] == "new"
                          else srv.submit_continuation(tickets[sp[1]], sp[2]))
        done = []
        for i in range(m):
            img, st = srv.wait(tickets[i])
            lat[i] = st["latency_ms"]
            done.append(start + arrivals[i] + st["latency_ms"] / 1000.0)
            if rate == args.serve_rates[0] and len(images) < args.serve_check:
                images[i] = img
        makespan = max(done) - (start + arrivals[0])
        for t in tickets:
            srv.release(t)
        runs.append({"rate_per_s": rate, "requests": m, "continuations": sum(1 for s in spec[:m] if s[0] == "cont"),
                     "arrival_window_s": float(arrivals[-1]), "samples": int(sum(samples[:m])),
                     "makespan_s": makespan, "samples_per_s": sum(samples[:m]) / makespan, **percentiles(lat),
                     "_arrivals": arrivals})
    st = srv.stats()
    srv.close()
    # The plain path: measured service time of every request, in order.
    m_all = max(r["requests"] for r in runs)
    need = {sp[1] for sp in spec[:m_all] if sp[0] == "cont"}
    renderers, service, identical = {}, [], []
    shared = api.PathTraceCudaRenderer(ctx)
    for i in range(m_all):
        sp = spec[i]
        torch.cuda.synchronize()
        if sp[0] == "new":
            s, _, e = scenes[sp[1]]
            # A request that a continuation will extend keeps its own
            # renderer (its accumulator); the others share one.
            r = api.PathTraceCudaRenderer(ctx) if i in need else shared
            r.tracer_mut().set_environment(api.EnvironmentMap(e) if e is not None else None)
            t0 = time.perf_counter()
            img = r.render_hdr(s, sp[2])
            service.append(time.perf_counter() - t0)
            if i in need:
                renderers[i] = r
        else:
            r = renderers[sp[1]]
            t0 = time.perf_counter()
            r.tracer.refine(sp[2])
            img = r.tracer.hdr()
            service.append(time.perf_counter() - t0)
        if i in images:
            identical.append(bool(np.array_equal(img, images[i])))
    for r in list(renderers.values()) + [shared]:
        r.tracer.close()
    for run in runs:
        arr = run.pop("_arrivals")
        m = run["requests"]
        free_at, plat, end = 0.0, [], 0.0
        for a, s_ in zip(arr, service[:m]):
            free_at = max(a, free_at) + s_
            plat.append(1000.0 * (free_at - a))
        plain_sps = sum(samples[:m]) / (free_at - arr[0])
        run["plain"] = {"samples_per_s": plain_sps, **percentiles(plat)}
        run["speedup_vs_plain"] = run["samples_per_s"] / plain_sps
    plain_busy = sum(samples[:m_all]) / sum(service)
    return {"scenes": len(scenes), "budget_gb": args.serve_budget_gb, "scene_gen_s": gen_s,
            "register_s": register_s, "scene_uploads": st["scene_uploads"], "scene_evictions": st["scene_evictions"],
            "peak_resident_gb": st["peak_resident_bytes"] / (1 << 30), "waves": st["waves"],
            "gpu_mrays_per_s": st["rays"] / (st["gpu_ms"] / 1000.0) / 1e6 if st["gpu_ms"] > 0 else None,
            "runs": runs,
            "plain_service_samples_per_s": plain_busy,
            "plain_call": "new: PathTraceCudaRenderer.render_hdr (scene prepared + uploaded per call); "
                          "continuation: refine(16) + hdr on its base request's renderer",
            "bit_identical_checked": len(identical), "bit_identical": all(identical) if identical else None}


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


def profiled_l2(kernel: str, config: str, wave_paths: int):
    """L2 figures of `kernel` from the committed ncu summary (lines
    `l2_bytes_per_launch | N` and `l2_pct_of_peak | X`): the L2 traffic
    (lts__t_sectors x 32 B) per launch, scaled like the DRAM traffic, and the
    L2 throughput as a share of its peak (the traversal kernels' tree and
    records live in L2, so this is their nearer bound)."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_*.md"))):
        text = open(path).read()
        if f"config={config}" not in text:
            continue
        b = re.search(r"l2_bytes_per_launch \| (\d+)", text)
        pct = re.search(r"l2_pct_of_peak \| ([0-9.]+)", text)
        if not b and not pct:
            continue
        w = re.search(r"profiled_wave_paths \| (\d+)", text)
        scale = wave_paths / int(w.group(1)) if w else 1.0
        return {"bytes_per_launch": int(int(b.group(1)) * scale) if b else None,
                "pct_of_peak": float(pct.group(1)) if pct else None,
                "source": os.path.relpath(path, ROOT)}
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


def oracle_mixed(reqs, passes: int = 0, budget_s: float = 0.0, first_pass: int = 0, stride: int = 256):
    """The oracle (CPU restatement of the reference) over the request mix on
    all host cores. Pass p renders, of every request r, the rows
    y = (17 r + p) mod `stride` + k * `stride` at the request's full spp: each
    pass is about 1/`stride` of the whole mix, in the mix's own proportions
    of scenes, sizes, spp and bounces. Rows run in parallel, one host thread
    each. Runs `passes` passes, or as many as fit in `budget_s`. Returns
    (camera paths, seconds per pass, rays, cores)."""
    import concurrent.futures as cf
    orc = entry.load_oracle()
    from oxideav_render_b200.scene import Camera
    cores = os.cpu_count() or 1
    built = {}
    jobs = []
    for k, s, o, env in reqs:
        if k not in built:
            desc = s.to_desc(o)
            built[k] = (desc, orc.OracleScene(desc), orc.OracleEnv(env) if env is not None else None)
        _, sc, oenv = built[k]
        jobs.append((sc, Camera.resolve(s, o, o.width, o.height), o, oenv))

    def one(job, row):
        sc, cam, o, oenv = job
        _, rc = orc.refine_rows(sc, cam, o, oenv, row, 1, 1, 0, o.path_trace.samples_per_pixel, 1)
        return o.width * o.path_trace.samples_per_pixel, rc[0] + rc[1]

    times, paths, rays = [], 0, 0
    with cf.ThreadPoolExecutor(cores) as ex:
        p = first_pass
        t_start = time.perf_counter()
        while (passes and len(times) < passes) or (not passes and time.perf_counter() - t_start < budget_s):
            t0 = time.perf_counter()
            work = [(job, y) for r, job in enumerate(jobs)
                    for y in range((17 * r + p) % stride, job[2].height, stride)]
            # Largest rows first: the pool ends each pass with small ones.
            work.sort(key=lambda jy: -jy[0][2].width * jy[0][2].path_trace.samples_per_pixel)
            for f in [ex.submit(one, job, y) for job, y in work]:
                n, r = f.result()
                paths += n
                rays += r
            times.append(time.perf_counter() - t0)
            p += 1
    return paths, times, rays, cores


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
    """The reference arm: the oracle (the CPU restatement of the reference's
    PathTracer; the Rust crate cannot be built here) on the host cores, on
    the headline's request mix. One step = one pass: every 256th row of
    every request at its full spp (a bounded sample of the mix, in its
    proportions)."""
    ws, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    entry.load_package()
    reqs = mixed_requests(args.mixed, 2026)
    oracle_mixed(reqs, passes=args.warmup)  # warm-up passes (also builds the oracle scenes)
    paths, times, rays, cores = oracle_mixed(reqs, passes=args.steps, first_pass=args.warmup)
    value = paths / sum(times)
    sample = (f"every 256th row of each of the {len(reqs)} requests per step (offset by request and step) at the "
              f"request's full spp, about 1/256 of the mix; {paths // max(len(times), 1)} camera paths per step")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": MIX_WORKLOAD, "parallelism": "host threads"},
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


MIX_WORKLOAD = ("config 3 request mix: 64 requests (seed 2026), scene uniform over {Cornell box C0, sphere grid C1, "
                "stress scene C2 (~4.1M tris, env + 8 emitters), 8 random soups of 10k-500k tris}, resolution "
                "{128^2, 256^2, 512^2, 1024x768}, spp {1, 4, 16, 64}, bounces {2, 4, 8}")


def stage_roofline(bc, peak, peak_kind, config_tag, wave_paths):
    """Roofline of the dominant wavefront stage from a stage-timed refine:
    its algorithmic bytes (the byte model) / its device time."""
    ext, shadow = bc["ext_rays"], bc["shadow_rays"]
    stage = bc["stage_ms"]
    stage_bytes = {
        "extend": 48 * ext + 64 * bc["ext_nodes"] + 48 * bc["ext_tris"],
        "shadow": 48 * shadow + 64 * bc["sh_nodes"] + 48 * bc["sh_tris"],
        # Per shaded vertex: hit (t, barycentrics, id: 20 B), path state read
        # (7 x 16 B) and written back (5 x 16 B), the triangle's corner
        # positions and normals (2 x 36 B) and material / flag word (8 B), the
        # NEE kernel's precomputed sample (16 B read), queue traffic (3 x 4 B);
        # per shadow ray written: origin, direction, contribution (48 B).
        "shade": ext * (20 + 112 + 80 + 72 + 8 + 16 + 12) + 48 * shadow,
        # Per vertex: hit and seeds read (36 B), corner positions (36 B),
        # previous vertex (16 B), the sample written (48 B).
        "nee": ext * (36 + 36 + 16 + 48),
        "megakernel": algorithmic_bytes(ext, shadow, bc["ext_nodes"] + bc["sh_nodes"],
                                        bc["ext_tris"] + bc["sh_tris"], 0),
        "accumulate": 32 * bc["samples"],
    }
    names = {"extend": "k_wf_extend", "shade": "k_wf_shade", "shadow": "k_wf_shadow", "megakernel": "k_megakernel",
             "accumulate": "k_accumulate", "nee": "k_wf_nee"}
    dom = max((k for k in stage_bytes if stage.get(k, 0) > 0), key=lambda k: stage[k])
    launches = bc["rounds"] if dom in ("extend", "shade", "shadow", "nee") else bc["waves"]
    achieved = stage_bytes[dom] / (stage[dom] / 1000.0) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": profiled_traffic(names[dom], config_tag, wave_paths), "peak_kind": peak_kind,
            "kernel": names[dom], "bytes_per_launch": stage_bytes[dom] / max(launches, 1),
            "ms_per_launch": stage[dom] / max(launches, 1), "launches": int(launches),
            "l2": profiled_l2(names[dom], config_tag, wave_paths),
            "stage_share": stage[dom] / max(sum(v for v in stage.values() if v > 0), 1e-9)}


def run_frame(ctx, api, torch, args, ws, rank, flush):
    """Secondary: one plain frame of --config (default: the C1 sphere grid,
    512^2, 256 spp) refined by one tracer on a resident scene, K steps, plus
    its end-to-end one-shot render and raycast frames of the same scene."""
    scene, opts, env, wname = workload(args.config)
    if args.spp:
        opts = opts.replace(path_trace=opts.path_trace.__class__(**{**opts.path_trace.__dict__,
                                                                   "samples_per_pixel": args.spp}))
        wname += f" (override: {args.spp} spp)"
    spp = opts.path_trace.samples_per_pixel
    samples_per_step = opts.width * opts.height * spp
    if args.seed_per_rank and ws > 1:
        opts = opts.replace(path_trace=opts.path_trace.__class__(**{**opts.path_trace.__dict__, "seed": rank}))
    tracer = api.PathTracer(ctx)
    if env is not None:
        tracer.set_environment(api.EnvironmentMap(env))
    tracer.sync(scene, opts)
    tuned = None
    if args.autotune:
        t0 = time.perf_counter()
        tuned = ctx.autotune(tracer, 0)
        tuned["seconds"] = time.perf_counter() - t0
    for _ in range(args.warmup):
        tracer.refine(spp)
    barrier(ws)
    kernel_ms, ext, shadow = [], 0, 0
    for _ in range(args.frame_steps):
        flush.zero_()
        torch.cuda.synchronize()
        tracer.refine(spp)
        kernel_ms.append(tracer.last_kernel_ms())
        e, s = tracer.ray_counts()
        ext, shadow = ext + e, shadow + s
    barrier(ws)
    ctx.set_stage_timing(True)
    flush.zero_()
    torch.cuda.synchronize()
    tracer.refine(spp)
    bc = api.batch_counters(ctx)
    ctx.set_stage_timing(False)
    dev_s = max_over_ranks(sum(kernel_ms) / 1000.0, ws)
    peak, peak_kind = load_peaks()
    wave_slots = (tuned or {}).get("wave_slots") or args.wave_slots or (1 << 23)
    out = {"workload": wname, "samples_per_step": samples_per_step, "steps": args.frame_steps,
           "value": samples_per_step * args.frame_steps * ws / dev_s, "unit": "samples/s",
           "ms_per_step": 1000 * dev_s / args.frame_steps,
           "mrays_per_s": (ext + shadow) / (sum(kernel_ms) / 1000.0) / 1e6,
           "stage_ms_per_frame": {k: v for k, v in bc["stage_ms"].items() if v > 0},
           "roofline": stage_roofline(bc, peak, peak_kind, args.config, min(wave_slots, samples_per_step)),
           "autotuned": tuned,
           "l2": "flushed (256 MB write) before every timed step"}
    renderer = api.PathTraceCudaRenderer(ctx)
    if env is not None:
        renderer.tracer_mut().set_environment(api.EnvironmentMap(env))
    # One untimed call, then the median of five: a call's host-side
    # preparation varies from call to call (allocation, page faults), and the
    # upload's own split is recorded per call.
    e2e_s, uploads = [], []
    for i in range(6):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        img = renderer.render(scene, opts)
        if i > 0:
            e2e_s.append(time.perf_counter() - t0)
            uploads.append(ctx.upload_seconds(renderer.tracer.scene_id))
    e2e_t = max_over_ranks(statistics.median(e2e_s), ws)
    up = {k: round(1000 * statistics.median(u[k] for u in uploads), 2) for k in uploads[0]}
    out["e2e"] = {"value": samples_per_step * ws / e2e_t, "unit": "samples/s", "ms_per_step": 1000 * e2e_t,
                  "walls_ms": [round(1000 * t, 1) for t in e2e_s], "wall_stat": "median",
                  "upload_ms_median": up,
                  "h2d_bytes_per_step": int(ctx.scene_bytes(renderer.tracer.scene_id)),
                  "d2h_bytes_per_step": int(img.nbytes),
                  "call": "PathTraceCudaRenderer.render (scene preparation and upload incl. the BVH build, "
                          "refine, sRGB image readback)"}
    renderer.tracer.close()
    if args.raycast:
        out["raycast"] = run_raycast(ctx, api, torch, scene, opts, cpu=rank == 0 and not args.no_cpu_baseline)
        out["raycast_pbr"] = run_raycast(ctx, api, torch, scene, opts, cpu=rank == 0 and not args.no_cpu_baseline,
                                         pbr=True)
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(scene, opts, env, args.cpu_seconds / 2)
    tracer.close()
    return out


def run_b200(args):
    import torch
    ws, rank, local = dist_setup()
    entry.load_package()
    from oxideav_render_b200 import api
    ctx = api.Context(local if ws > 1 else torch.cuda.current_device())
    if not args.wave_overlap:
        ctx.set_wave_overlap(False)
    elif args.wave_arenas:
        ctx.set_wave_overlap(args.wave_arenas)
    if args.wave_slots:
        ctx.set_wave_slots(args.wave_slots)
    if args.schedule == "megakernel":
        ctx.set_schedule(0)
    if args.trav_threads or args.claim_chunk:
        ctx.set_traversal(args.trav_threads or 256, args.claim_chunk or 1)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    if args.mixed == 0:
        # Profiling case: the single frame of --config alone.
        frame = run_frame(ctx, api, torch, args, ws, rank, flush)
        if rank == 0:
            print(json.dumps(frame))
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    # Headline: the config-3 request mix in shared waves (one tracer per
    # request, scenes resident). With N ranks the mix holds 64 N requests
    # (seed 2026; request i renders with sample seed i) and rank r serves
    # requests r, r + N, ... with its own scene cache: 64 requests per GPU
    # (weak scaling), no exchange. N = 1 is exactly the 64-request mix.
    from oxideav_render_b200 import shard
    reqs = shard.shard(mixed_requests(args.mixed * ws, 2026), rank, ws)
    tracers, b = run_batched(ctx, api, torch, reqs, args, ws, flush)
    dev_s = max_over_ranks(sum(b["ms"]) / 1000.0, ws)
    value = b["total"] * args.steps * ws / dev_s
    peak, peak_kind = load_peaks()
    bc = b["counters"]
    roofline = stage_roofline(bc, peak, peak_kind, "mixed", min(args.wave_slots or (1 << 23), b["total"]))
    launches = args.steps * (2 * bc["waves"] + 8 * bc["rounds"])

    # End to end on the same requests through the serving C ABI (host I/O).
    e2e = run_served_batch(ctx, api, torch, reqs, args, tracers)
    e2e_wall = max_over_ranks(e2e["ms_per_step"] / 1000.0, ws)
    e2e["value"] = b["total"] * ws / e2e_wall
    e2e["ms_per_step"] = 1000 * e2e_wall
    # The plain per-request path on the same requests.
    plain = run_plain_requests(ctx, api, torch, reqs, tracers)
    for t in tracers:
        t.close()
    for sid in b["scene_ids"].values():
        ctx.release(sid)
    vs_plain = {
        "same_requests": True,
        "plain_one_shot_samples_per_s": plain["one_shot"]["samples_per_s"],
        "plain_resident_samples_per_s": plain["resident"]["samples_per_s"],
        "served_e2e_samples_per_s": e2e["value"] / ws,
        "batched_device_samples_per_s": value / ws,
        "speedup_served_vs_plain_one_shot": (e2e["value"] / ws) / plain["one_shot"]["samples_per_s"],
        "speedup_served_vs_plain_resident": (e2e["value"] / ws) / plain["resident"]["samples_per_s"],
        "speedup_batched_vs_plain_resident": (value / ws) / plain["resident"]["samples_per_s"],
        "latency_ms": {"served": {"p50": e2e["p50_ms"], "p99": e2e["p99_ms"]},
                       "plain_one_shot": {"p50": plain["one_shot"]["p50_ms"], "p99": plain["one_shot"]["p99_ms"]},
                       "plain_resident": {"p50": plain["resident"]["p50_ms"], "p99": plain["resident"]["p99_ms"]}},
        "latency_note": "all requests submitted at once; plain latencies are cumulative, in request order",
        "per_rank": ws > 1,
    }

    frame = run_frame(ctx, api, torch, args, ws, rank, flush) if args.frame else None
    poisson = run_poisson(ctx, api, torch, args) if (args.serve_rates and ws == 1) else None
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        paths, times, rays, cores = oracle_mixed(reqs, budget_s=args.cpu_seconds)
        cpu = {"value": paths / sum(times), "unit": "samples/s", "cores": cores, "kind": "port",
               "sample": f"{len(times)} passes over every 256th row of each of the {len(reqs)} requests at "
                         f"its full spp ({paths} camera paths, {sum(times):.1f} s)",
               "mrays_per_s": rays / sum(times) / 1e6}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": MIX_WORKLOAD, "requests_per_step": len(reqs), "samples_per_step": b["total"],
                       "global_batch": b["total"] * ws,
                       "parallelism": f"request mix per rank x{ws}" if ws > 1 else "single GPU",
                       "path": "pt_tracer_refine_many: every request's paths in shared wavefront waves",
                       "resident_bvh": "spatial-split (host build once per scene)" if args.spatial_bvh
                       else "binned SAH", "scene_upload_s": b["scene_upload_s"],
                       "l2": "flushed (256 MB write) before every timed step; resident scenes 2+ GB",
                       "schedule": args.schedule},
            "mrays_per_s": b["rays"] / (sum(b["ms"]) / 1000.0) / 1e6,
            "waves_per_step": b["waves"] / args.steps,
            "stage_ms_per_step": {k: v for k, v in bc["stage_ms"].items() if v > 0},
            "stage_note": "stage split from one extra batch timed stage by stage (sequential waves)",
            "roofline": roofline,
            "e2e": e2e,
            "vs_plain": vs_plain,
            "served_poisson": poisson,
            "plain_frame": frame,
            "cpu_baseline": cpu,
            "clocks": b["clocks"],
            "gpu_launches": int(launches),
        }
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mixed", type=int, default=64,
                    help="requests of the headline request mix (0: only the single frame of --config, for profiling)")
    ap.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "soup"],
                    help="scene of the secondary single-frame measurement")
    ap.add_argument("--no-frame", dest="frame", action="store_false", help="skip the single-frame measurement")
    ap.add_argument("--frame-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed-per-rank", action="store_true")
    ap.add_argument("--spp", type=int, default=0, help="override the frame's samples per pixel (profiling cases)")
    ap.add_argument("--schedule", default="wavefront", choices=["megakernel", "wavefront"])
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default configuration instead of pt_autotune's per-class choice (frame only)")
    ap.add_argument("--serve-rates", default="5,200",
                    help="Poisson arrival rates (requests/s) of the config-4 runs, comma-separated ('' : skip)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="arrival window per config-4 run")
    ap.add_argument("--serve-max", type=int, default=300, help="requests per config-4 run at most")
    ap.add_argument("--serve-scenes", type=int, default=32, help="resident scenes of the config-4 runs")
    ap.add_argument("--serve-budget-gb", type=float, default=60.0, help="HBM budget of the resident scenes")
    ap.add_argument("--serve-check", type=int, default=8, help="served images compared with the plain path")
    ap.add_argument("--serve-wave-slots", type=int, default=0, help="path slots per served wave (0: the server's default)")
    ap.add_argument("--serve-depth", type=int, default=0, help="served waves in flight (0: the server's default)")
    ap.add_argument("--binned-bvh", dest="spatial_bvh", action="store_false",
                    help="resident and served scenes get the binned-SAH tree instead of the spatial-split one")
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
    ap.add_argument("--trav-threads", type=int, default=0, help="traversal block size 128 / 256 (0: default)")
    ap.add_argument("--claim-chunk", type=int, default=0, help="queue entries per traversal refill 1 / 2 / 4 (0: default)")
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
