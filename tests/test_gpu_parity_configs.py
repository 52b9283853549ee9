"""Image parity on the benchmark configurations themselves, at their full
geometry, resolution and sample counts, against the oracle (the CPU
restatement of the reference's PathTracer):

* config 1, the metallic x roughness sphere grid: 512x512, 256 spp, 8
  bounces, the 200,706-triangle scene with its textured floor;
* config 2, the stress scene: 1920x1080, 64 spp, 8 bounces, the ~4.1 M
  triangle heightfield + 500 spheres (diffuse / metal / dielectric /
  clearcoat), 8 emissive triangles (f64 spherical-triangle sampling) and a
  512x256 environment map.

The GPU renders the whole frame; the oracle renders evenly strided rows of
the same frame (the sample streams are keyed by pixel and sample index, so
the rows are the same estimates). Bars: per-pixel MAE <= 2e-3 and PSNR >=
45 dB (peak 1.0) over those rows.

Then the statistical bar: region means of 16,384-spp renders must lie
within 3 sigma of the oracle's. Here the GPU and the oracle use DIFFERENT
seeds, so the two renders are independent estimates of the same image and
the test checks that they converge to the same values (no bias), not only
that they share samples. Sigma per region and channel comes from 16
batches of 1,024 spp on each side: the standard error of the batch means,
combined over both renders. The seeds are fixed, so the outcome is
deterministic. The reference's region metrics are testscenes.rs:1103-1138;
its convergence test is pathtrace.rs:3447-3463.
"""
import os

import numpy as np
import pytest

from oxideav_render_b200 import api, testscenes as ts
from oxideav_render_b200.options import PathTraceOptions
from oxideav_render_b200.scene import Camera

pytestmark = pytest.mark.gpu

MAE_MAX = 2e-3
PSNR_MIN = 45.0
CORES = os.cpu_count() or 1


def resolve_rows(acc: np.ndarray) -> np.ndarray:
    """Covered mean per pixel (what PathTracer::hdr shows for covered pixels)."""
    n = np.maximum(acc[..., 3:4], 1.0)
    return (acc[..., :3] / n).astype(np.float32)


def strided_parity(oracle, ctx, scene, opts, env, stride):
    w, h, spp = opts.width, opts.height, opts.path_trace.samples_per_pixel
    t = api.PathTracer(ctx)
    if env is not None:
        t.set_environment(api.EnvironmentMap(env))
    t.sync(scene, opts)
    t.refine(spp)
    full = t.accum()
    t.close()
    row0 = stride // 2
    rows = list(range(row0, h, stride))
    desc = scene.to_desc(opts)
    sc = oracle.OracleScene(desc)
    cam = Camera.resolve(scene, opts, w, h)
    oenv = oracle.OracleEnv(env) if env is not None else None
    acc, _ = oracle.refine_rows(sc, cam, opts, oenv, row0, stride, len(rows), 0, spp, CORES)
    g = resolve_rows(full[rows])
    o = resolve_rows(acc)
    # Coverage (the alpha of the covered mean) must agree exactly.
    assert np.array_equal(full[rows][..., 3], acc[..., 3])
    return ts.hdr_mae(g, o), ts.hdr_psnr(g, o), len(rows)


def test_parity_config1_full_frame(oracle, ctx):
    scene, opts = ts.sphere_grid_c1(512, 256)
    mae, psnr, n = strided_parity(oracle, ctx, scene, opts, None, stride=32)
    assert n == 16
    assert mae <= MAE_MAX and psnr >= PSNR_MIN, (mae, psnr)


def test_parity_config2_full_geometry(oracle, ctx):
    scene, opts, env = ts.stress_c2()
    assert scene.triangle_count() > 4_000_000
    mae, psnr, n = strided_parity(oracle, ctx, scene, opts, env, stride=120)
    assert n == 9
    assert mae <= MAE_MAX and psnr >= PSNR_MIN, (mae, psnr)


# ----------------------------------------------------------------------------- 16k-spp region means

BATCHES, BATCH_SPP = 16, 1024  # 16,384 spp


def batch_region_means(refine, read_accum, regions):
    """Region means of each batch's image (RGB) -> (batches, regions, 3)."""
    prev = None
    out = []
    for _ in range(BATCHES):
        refine(BATCH_SPP)
        acc = read_accum()
        batch = acc if prev is None else acc - prev
        prev = acc.copy()
        img = batch[..., :3] / np.maximum(batch[..., 3:4], 1.0)
        out.append([img[y0:y1, x0:x1].reshape(-1, 3).mean(axis=0) for (x0, y0, x1, y1) in regions])
    return np.asarray(out)


def region_check(oracle, ctx, scene, opts, env, gpu_seed, oracle_seed, block):
    w, h = opts.width, opts.height
    regions = [(x, y, x + block, y + block) for y in range(0, h, block) for x in range(0, w, block)]
    og = opts.replace(path_trace=PathTraceOptions(**{**opts.path_trace.__dict__, "seed": gpu_seed}))
    oo = opts.replace(path_trace=PathTraceOptions(**{**opts.path_trace.__dict__, "seed": oracle_seed}))
    t = api.PathTracer(ctx)
    if env is not None:
        t.set_environment(api.EnvironmentMap(env))
    t.sync(scene, og)
    g = batch_region_means(t.refine, t.accum, regions)
    t.close()
    desc = scene.to_desc(oo)
    sc = oracle.OracleScene(desc)
    cam = Camera.resolve(scene, oo, w, h)
    ot = oracle.OracleTracer(sc, cam, oo, oracle.OracleEnv(env) if env is not None else None, CORES)
    o = batch_region_means(ot.refine, lambda: ot.accum, regions)
    mg, mo = g.mean(axis=0), o.mean(axis=0)
    se = np.sqrt(g.var(axis=0, ddof=1) / BATCHES + o.var(axis=0, ddof=1) / BATCHES)
    z = np.abs(mg - mo) / np.maximum(se, 1e-12)
    return z, mg, mo, se


@pytest.mark.parametrize("case", ["cornell", "spheres", "env_emitters"])
def test_region_means_of_16k_spp_renders_within_3_sigma(oracle, ctx, case):
    if case == "cornell":
        scene, opts = ts.cornell_c0()
        opts = opts.replace(width=16, height=16)
        env = None
    elif case == "spheres":
        scene, opts = ts.sphere_grid_c1(16, 1)
        env = None
    else:
        scene = ts.area_light_scene(0.35, 0.5)
        opts = ts.pt_opts(16, 1, 4)
        env = ts.env_noise(64, 32, np.random.default_rng(4))
    z, mg, mo, se = region_check(oracle, ctx, scene, opts, env, gpu_seed=11, oracle_seed=23, block=4)
    worst = np.unravel_index(np.argmax(z), z.shape)
    assert np.all(z <= 3.0), (case, worst, float(z.max()), mg[worst[0]], mo[worst[0]], se[worst[0]])
    # The comparison has power: the standard error is small against the signal.
    lit = mg > 1e-3
    assert np.median(se[lit] / mg[lit]) < 0.02, case
