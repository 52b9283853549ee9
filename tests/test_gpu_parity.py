"""GPU parity against the oracle (CPU restatement of the reference).

Bars (all through the C ABI):
  * sampler values and camera-ray hits (triangle id, t, barycentrics):
    bit-exact;
  * resolve (hdr / image) of a given accumulator: bit-exact;
  * BSDF eval / sample: relative error <= 2e-4 (device vs host libm
    transcendentals differ by ulps);
  * final HDR images at matched spp: mean absolute error <= 2e-3 and PSNR
    >= 45 dB (peak 1.0) over RGB.
"""
import math

import numpy as np
import pytest

from oxideav_render_b200 import api, testscenes as ts
from oxideav_render_b200.options import LightStrategy, PathTraceOptions
from oxideav_render_b200.scene import Camera

pytestmark = pytest.mark.gpu

MAE_MAX = 2e-3
PSNR_MIN = 45.0


def oracle_tracer(oracle, scene, opts, env=None):
    desc = scene.to_desc(opts)
    sc = oracle.OracleScene(desc)
    cam = Camera.resolve(scene, opts, max(opts.width, 1), max(opts.height, 1))
    t = oracle.OracleTracer(sc, cam, opts, env)
    t._keep = (desc, sc)
    return t


def gpu_tracer(ctx, scene, opts, env=None):
    t = api.PathTracer(ctx)
    if env is not None:
        t.set_environment(api.EnvironmentMap(env))
    t.sync(scene, opts)
    return t


def parity(oracle, ctx, scene, opts, env=None):
    spp = opts.path_trace.samples_per_pixel
    g = gpu_tracer(ctx, scene, opts, env)
    g.refine(spp)
    o = oracle_tracer(oracle, scene, opts, oracle.OracleEnv(env) if env is not None else None)
    o.refine(spp)
    a, b = g.hdr(), o.hdr()
    mae = ts.hdr_mae(a, b)
    psnr = ts.hdr_psnr(a, b)
    return mae, psnr, g, o


# ----------------------------------------------------------------------------- bit-exact stages


def test_sobol_values_bit_exact(oracle, ctx):
    for seed in [0, 1, 12345, 0xDEADBEEF]:
        dev = ctx.debug_sobol(4096, seed)
        ref = oracle.sobol_owen_4d_many(4096, seed)
        assert np.array_equal(dev, ref), seed


def test_sampler_patterns_bit_exact(oracle, ctx):
    scene, opts = ts.cornell_c0()
    opts = opts.replace(width=48, height=40, path_trace=PathTraceOptions(samples_per_pixel=4, seed=7))
    t = gpu_tracer(ctx, scene, opts)
    C = oracle.C
    out = np.zeros(4, np.float32)
    for index in [0, 3]:
        for pattern in [0, 1, 2, 9]:
            dev = t.debug_pattern(index, pattern)
            for y in range(0, 40, 3):
                for x in range(0, 48, 5):
                    oracle.lib().oracle_sampler_pattern(7, x, y, index, pattern,
                                                        out.ctypes.data_as(C.POINTER(C.c_float)))
                    assert np.array_equal(dev[y, x], out), (index, pattern, x, y)


def primary_parity(oracle, ctx, scene, opts, indices=(0, 1)):
    t = gpu_tracer(ctx, scene, opts)
    o = oracle_tracer(oracle, scene, opts)
    for index in indices:
        g_dev, tb = t.debug_primary_hits(index)
        g_ref, t_ref, b_ref = o.primary_hits(index)
        assert np.array_equal(g_dev, g_ref), f"triangle ids differ at {np.argwhere(g_dev != g_ref)[:5]}"
        hit = g_ref != 0xFFFFFFFF
        assert np.array_equal(tb[..., 0][hit], t_ref[hit])
        assert np.array_equal(tb[..., 1:][hit], b_ref[hit])
        assert hit.any()


def test_primary_hits_bit_exact_cornell_c0(oracle, ctx):
    scene, opts = ts.cornell_c0()
    primary_parity(oracle, ctx, scene, opts)


def test_primary_hits_bit_exact_sphere_grid_c1(oracle, ctx):
    scene, opts = ts.sphere_grid_c1(256, 4)
    primary_parity(oracle, ctx, scene, opts, indices=(0,))


def test_primary_hits_bit_exact_alpha_filters(oracle, ctx):
    # MASK cut-outs and stochastic BLEND coins in the any-hit filter.
    scene = ts.alpha_planes()
    primary_parity(oracle, ctx, scene, ts.pt_opts(64, 4, 2), indices=(0, 1, 2, 3))


def test_primary_hits_bit_exact_random_soup(oracle, ctx):
    scene = ts.random_soup(20000, seed=3)
    primary_parity(oracle, ctx, scene, ts.pt_opts(160, 2, 2), indices=(0,))


def test_resolve_is_bit_exact(oracle, ctx):
    scene, opts = ts.cornell_c0()
    from oxideav_render_b200.options import BackgroundColor, ToneMap
    for tm in [ToneMap.Clamp, ToneMap.Reinhard, ToneMap.AcesFitted]:
        o = opts.replace(width=64, height=64, tone_map=tm, exposure=1.7, background=BackgroundColor((30, 60, 90, 100)),
                         path_trace=PathTraceOptions(samples_per_pixel=8, max_bounces=3))
        t = gpu_tracer(ctx, scene, o)
        t.refine(8)
        acc = t.accum()
        ot = oracle_tracer(oracle, scene, o)
        ot.accum[...] = acc
        ot.samples = 8
        assert np.array_equal(t.hdr(), ot.hdr())
        assert np.array_equal(t.image(), ot.image())


# ----------------------------------------------------------------------------- BSDF


def test_device_bsdf_matches_oracle(oracle, ctx):
    import tests.test_oracle_bsdf as tb
    rng = np.random.default_rng(1)
    allc = [(n, m, f) for n, m, f in tb.cases(oracle)] + [(n, m, True) for n, m in tb.extension_cases(oracle)]
    for name, m, front in allc:
        v = tb.V / np.linalg.norm(tb.V)
        ng = tb.NG if front else -tb.NG
        dirs = rng.normal(size=(4096, 3)).astype(np.float32)
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        us = tb.sobol_u(oracle, 4096, 99)
        dev = ctx.debug_bsdf(m, v, ng, front, dirs, us)
        b = oracle.Bsdf(m, v, ng, front)
        f_ref, pdf_ref = b.eval_many(dirs)
        np.testing.assert_allclose(dev[:, :3], f_ref, rtol=2e-4, atol=1e-6, err_msg=name)
        np.testing.assert_allclose(dev[:, 3], pdf_ref, rtol=2e-4, atol=1e-6, err_msg=name)
        l_ref, fs_ref, ps_ref, ok_ref = b.sample_many(us)
        ok_dev = dev[:, 4] > 0.5
        assert np.mean(ok_dev == ok_ref) > 0.995, name
        both = ok_dev & ok_ref
        np.testing.assert_allclose(dev[both, 5:8], l_ref[both], atol=2e-4, err_msg=name)


# ----------------------------------------------------------------------------- images


def test_hdr_parity_cornell_c0(oracle, ctx):
    scene, opts = ts.cornell_c0()
    mae, psnr, g, _ = parity(oracle, ctx, scene, opts)
    assert mae <= MAE_MAX and psnr >= PSNR_MIN, (mae, psnr)


def test_hdr_parity_sphere_grid_c1_reduced(oracle, ctx):
    scene, opts = ts.sphere_grid_c1(128, 16)
    mae, psnr, _, _ = parity(oracle, ctx, scene, opts)
    assert mae <= MAE_MAX and psnr >= PSNR_MIN, (mae, psnr)


def test_hdr_parity_material_extensions(oracle, ctx):
    scene = ts.material_extensions()
    opts = ts.pt_opts(96, 16, 6)
    mae, psnr, _, _ = parity(oracle, ctx, scene, opts)
    assert mae <= MAE_MAX and psnr >= PSNR_MIN, (mae, psnr)


def test_hdr_parity_environment_and_emitters(oracle, ctx):
    scene = ts.area_light_scene(0.35, 0.5)
    rng = np.random.default_rng(4)
    env = ts.env_noise(64, 32, rng)
    for s in [LightStrategy.Mis, LightStrategy.LightOnly, LightStrategy.BsdfOnly]:
        mae, psnr, _, _ = parity(oracle, ctx, scene, ts.pt_opts(48, 16, 4, strategy=s), env)
        assert mae <= MAE_MAX and psnr >= PSNR_MIN, (s, mae, psnr)


def test_hdr_parity_alpha_and_glass(oracle, ctx):
    for scene, o in [(ts.alpha_planes(), ts.pt_opts(48, 8, 4)), (ts.glass_scene(True), ts.pt_opts(32, 16, 8)),
                     (ts.dispersive_sphere(1.0), ts.pt_opts(48, 8, 8))]:
        mae, psnr, _, _ = parity(oracle, ctx, scene, o)
        assert mae <= MAE_MAX and psnr >= PSNR_MIN, (mae, psnr)


# ----------------------------------------------------------------------------- reference known answers on the GPU


def gpu_hdr(ctx, scene, opts, env=None):
    t = gpu_tracer(ctx, scene, opts, env)
    t.refine(opts.path_trace.samples_per_pixel)
    return t.hdr()


def mean_rgb(img):
    return img[..., :3].astype(np.float64).mean(axis=(0, 1))


def test_gpu_white_furnace(ctx):
    scene = ts.furnace_scene(0.5, 1.0)
    for s in [LightStrategy.Mis, LightStrategy.LightOnly, LightStrategy.BsdfOnly]:
        m = mean_rgb(gpu_hdr(ctx, scene, ts.pt_opts(8, 64, 64, strategy=s)))
        assert np.all(np.abs(m - 2.0) < 0.04), (s, m)


def test_gpu_glass_point_light_and_clamp(ctx):
    thin = mean_rgb(gpu_hdr(ctx, ts.glass_scene(False), ts.pt_opts(4, 16, 8)))[0]
    vol = mean_rgb(gpu_hdr(ctx, ts.glass_scene(True), ts.pt_opts(4, 16, 8)))[0]
    assert abs(thin - 0.92) < 0.03 and abs(vol - 0.46) < 0.03, (thin, vol)
    l = mean_rgb(gpu_hdr(ctx, ts.point_light_plane(), ts.pt_opts(2, 4, 1)))[0]
    assert abs(l - 4.0 / math.pi) < 0.01, l
    c = mean_rgb(gpu_hdr(ctx, ts.point_light_plane(), ts.pt_opts(2, 4, 1, clamp=0.5)))[0]
    assert abs(c - 0.5) < 1e-3, c


def test_gpu_uniform_environment(ctx):
    scene = ts.lambert_plane(0.5)
    env = np.ones((8, 16, 4), np.float32)
    for s in [LightStrategy.Mis, LightStrategy.LightOnly, LightStrategy.BsdfOnly]:
        m = mean_rgb(gpu_hdr(ctx, scene, ts.pt_opts(6, 64, 2, strategy=s), env))
        assert abs(m[0] - 0.5) < 0.02, (s, m)
