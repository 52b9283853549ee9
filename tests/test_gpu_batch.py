"""Batched refine: many tracers in shared waves end bit-identical to
refining each tracer alone (different scenes, resolutions, spp, bounce
limits, environment maps; both schedules; waves that split images)."""
import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import PathTraceOptions

pytestmark = pytest.mark.gpu


def make_requests():
    rng = np.random.default_rng(11)
    c0, o0 = ts.cornell_c0()
    c1, o1 = ts.sphere_grid_c1(64, 2)
    soup = ts.random_soup(5000, seed=2)
    env = ts.env_noise(32, 16, rng)
    return [
        (c0, o0.replace(width=48, height=40, path_trace=PathTraceOptions(samples_per_pixel=5, max_bounces=8)), None),
        (c1, o1.replace(path_trace=PathTraceOptions(samples_per_pixel=3, max_bounces=4)), None),
        (soup, ts.pt_opts(33, 7, 2, h=21), None),
        (ts.area_light_scene(0.35, 0.5), ts.pt_opts(24, 4, 3), env),
        (ts.material_extensions(), ts.pt_opts(40, 2, 6), None),
        (c0, o0.replace(width=17, height=9, path_trace=PathTraceOptions(samples_per_pixel=9, max_bounces=2, seed=5)),
         None),
    ]


def tracer_for(ctx, scene, opts, env):
    t = api.PathTracer(ctx)
    if env is not None:
        t.set_environment(api.EnvironmentMap(env))
    t.sync(scene, opts)
    return t


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("slots", [1 << 22, 3000])
def test_batched_refine_is_bit_identical_to_separate_refines(ctx, schedule, slots):
    ctx.set_schedule(schedule)
    ctx.set_wave_slots(slots)
    try:
        reqs = make_requests()
        alone = []
        for scene, opts, env in reqs:
            t = tracer_for(ctx, scene, opts, env)
            t.refine(opts.path_trace.samples_per_pixel)
            alone.append(t.accum())
            t.close()
        tracers = [tracer_for(ctx, s, o, e) for s, o, e in reqs]
        # Two batched calls: progressive continuation inside the batch too.
        first = [max(o.path_trace.samples_per_pixel // 2, 1) for _, o, _ in reqs]
        api.refine_many(ctx, tracers, first)
        api.refine_many(ctx, tracers, [o.path_trace.samples_per_pixel - f for (_, o, _), f in zip(reqs, first)])
        for t, ref, (_, o, _) in zip(tracers, alone, reqs):
            assert t.samples() == o.path_trace.samples_per_pixel
            assert np.array_equal(t.accum(), ref)
        st = api.batch_stats(ctx)
        assert st["waves"] >= 1 and st["rays"] > 0
        for t in tracers:
            t.close()
    finally:
        ctx.set_schedule(abi.PT_SCHEDULE_WAVEFRONT)
        ctx.set_wave_slots(abi.PT_DEFAULT_WAVE_SLOTS)


def test_batch_rejects_duplicate_tracers(ctx):
    scene, opts = ts.cornell_c0()
    t = tracer_for(ctx, scene, opts.replace(width=8, height=8), None)
    with pytest.raises(api.RenderError):
        api.refine_many(ctx, [t, t], [1, 1])
    t.close()
