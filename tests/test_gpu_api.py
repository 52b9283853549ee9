"""PathTracer / PathTraceCudaRenderer semantics on the GPU (ports of
src/pathtrace.rs:3566-3626 and the robustness tests of src/lib.rs:385-655)."""
import ctypes as C

import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import (BackgroundColor, CameraSpec, PathTraceOptions, Projection, RenderBackend,
                                         ToneMap)
from oxideav_render_b200.scene import PreparedScene, Primitive

pytestmark = pytest.mark.gpu


def test_renders_are_deterministic_and_refinement_is_additive(ctx):
    scene = ts.area_light_scene(0.5, 0.0)
    o = ts.pt_opts(9, 8, 4)
    r = api.PathTraceCudaRenderer(ctx)
    a = r.render_hdr(scene, o)
    b = api.PathTraceCudaRenderer(ctx).render_hdr(scene, o)
    assert np.array_equal(a, b)
    t = api.PathTracer(ctx)
    t.sync(scene, o)
    t.refine(3)
    t.refine(5)
    assert t.samples() == 8
    assert np.array_equal(t.hdr(), a), "refine(3)+refine(5) must equal refine(8)"
    assert not np.array_equal(api.PathTraceCudaRenderer(ctx).render_hdr(scene, ts.pt_opts(9, 8, 4, seed=1)), a)


def test_refinement_is_additive_across_waves(ctx):
    # Small waves split one refine into many launches; results are unchanged.
    scene, opts = ts.cornell_c0()
    o = opts.replace(width=40, height=30, path_trace=PathTraceOptions(samples_per_pixel=12, max_bounces=4))
    t1 = api.PathTracer(ctx)
    t1.sync(scene, o)
    t1.refine(12)
    ref = t1.accum()
    ctx.set_wave_slots(1024)
    try:
        t2 = api.PathTracer(ctx)
        t2.sync(scene, o)
        t2.refine(5)
        t2.refine(7)
        assert np.array_equal(t2.accum(), ref)
    finally:
        ctx.set_wave_slots(abi.PT_DEFAULT_WAVE_SLOTS)


@pytest.mark.parametrize("slots", [1024, 20000])
def test_overlapped_waves_are_bit_identical(ctx, slots):
    # Many small waves (traced two at a time in two arenas on two streams,
    # accumulated in wave order) against one wave at a time and the
    # megakernel: the same accumulators and ray counts, single tracers and a
    # batch of tracers of different scenes, sizes and bounce limits.
    cases = [ts.cornell_c0(), ts.sphere_grid_c1(48, 6)]
    cases[0] = (cases[0][0], cases[0][1].replace(width=40, height=30,
                                                 path_trace=PathTraceOptions(samples_per_pixel=12, max_bounces=6)))
    cases.append((ts.alpha_planes(), ts.pt_opts(24, 8, 3)))

    def run(schedule, overlap):
        ctx.set_schedule(schedule)
        ctx.set_wave_overlap(overlap)
        ctx.set_wave_slots(slots)
        try:
            ts_ = []
            for scene, o in cases:
                t = api.PathTracer(ctx)
                t.sync(scene, o)
                ts_.append(t)
            ts_[0].refine(5)
            api.refine_many(ctx, ts_, [7, 6, 8])
            out = [(t.accum(), t.ray_counts()) for t in ts_]
            for t in ts_:
                t.close()
            return out
        finally:
            ctx.set_wave_overlap(True)
            ctx.set_wave_slots(abi.PT_DEFAULT_WAVE_SLOTS)
            ctx.set_schedule(abi.PT_SCHEDULE_WAVEFRONT)

    mk = run(0, False)
    seq = run(1, False)
    ovl = run(1, True)
    ovl3 = run(1, 3)
    for (a, ra), (b, rb), (c, rc), (d, rd) in zip(mk, seq, ovl, ovl3):
        assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)
        assert ra == rb == rc == rd


def _accum_with(ctx, schedule, scene, opts, env=None):
    ctx.set_schedule(schedule)
    try:
        t = api.PathTracer(ctx)
        if env is not None:
            t.set_environment(api.EnvironmentMap(env))
        t.sync(scene, opts)
        t.refine(opts.path_trace.samples_per_pixel)
        out = t.accum(), t.ray_counts(), t.traversal_counts()
        t.close()
        return out
    finally:
        ctx.set_schedule(abi.PT_SCHEDULE_WAVEFRONT)


def _many_lights_scene() -> PreparedScene:
    """An emissive quad over a floor with a blocker, lit besides by a
    directional light, two range-limited point lights and two narrow spot
    lights: paths queue from zero to six shadow rays each (a light outside
    its range or cone adds none), so the shadow queue's rays per path vary
    from path to path."""
    from oxideav_render_b200.scene import directional_light, point_light, spot_light
    s = ts.area_light_scene(0.4, 0.3)
    grey = s.add_material(ts.diffuse_material((0.6, 0.6, 0.6), 0.8))
    s.add_primitive(ts.with_material(ts.cuboid([-0.3, 0.0, -0.3], [0.3, 0.5, 0.3]), grey))
    s.add_light(directional_light((1.0, 0.9, 0.8), 2.0), [0.0, 0.0, 0.0], [0.3, -1.0, 0.2])
    s.add_light(point_light((1.0, 0.2, 0.2), 6.0, range=1.5), [1.2, 0.8, 0.5], [0.0, -1.0, 0.0])
    s.add_light(point_light((0.2, 1.0, 0.2), 6.0, range=1.0), [-1.0, 0.6, -0.8], [0.0, -1.0, 0.0])
    s.add_light(spot_light((0.2, 0.2, 1.0), 9.0, inner=0.1, outer=0.3), [0.0, 1.8, 1.2], [0.0, -1.0, -0.5])
    s.add_light(spot_light((1.0, 1.0, 0.2), 9.0, range=3.0, inner=0.0, outer=0.2), [-1.5, 1.5, 0.0], [1.0, -1.0, 0.0])
    return s


@pytest.mark.parametrize("case", ["cornell", "spheres", "materials", "env", "alpha", "dispersion", "lights"])
def test_wavefront_schedule_is_bit_identical_to_megakernel(ctx, case):
    env = None
    if case == "lights":
        scene, opts = _many_lights_scene(), ts.pt_opts(64, 8, 5)
    elif case == "cornell":
        scene, opts = ts.cornell_c0()
        opts = opts.replace(width=96, height=80, path_trace=PathTraceOptions(samples_per_pixel=8, max_bounces=8))
    elif case == "spheres":
        scene, opts = ts.sphere_grid_c1(96, 4)
    elif case == "materials":
        scene, opts = ts.material_extensions(), ts.pt_opts(80, 4, 6)
    elif case == "env":
        scene, opts = ts.area_light_scene(0.35, 0.5), ts.pt_opts(48, 8, 4)
        env = ts.env_noise(64, 32, np.random.default_rng(4))
    elif case == "alpha":
        scene, opts = ts.alpha_planes(), ts.pt_opts(48, 8, 4)
    else:
        scene, opts = ts.dispersive_sphere(1.0), ts.pt_opts(48, 8, 8)
    # Host-built trees throughout: the traversal counts below compare
    # schedules on one tree.
    ctx.set_bvh_builder(abi.PT_BVH_BUILD_HOST)
    a, ra, ta = _accum_with(ctx, 0, scene, opts, env)
    try:
        # The wavefront on the two-child layout: the same tree, visited at
        # least as much (its speculative node phase may test boxes against
        # an older closest hit), identical hits.
        ctx.set_node_width(2, 2)
        b, rb, tb = _accum_with(ctx, 1, scene, opts, env)
        assert np.array_equal(a, b)
        assert ra == rb and tb[0] >= ta[0] and tb[1] >= ta[1]
        # On the four-child layout (either ray kind): other node visits,
        # identical hits.
        for ext, sh in ((4, 4), (2, 4), (4, 2)):
            ctx.set_node_width(ext, sh)
            c, rc, _ = _accum_with(ctx, 1, scene, opts, env)
            assert np.array_equal(a, c), (ext, sh)
            assert rc == ra
        # Material-sorted shading (the default) reorders work only.
        for sort in (False, True):
            ctx.set_material_sort(sort)
            d, rd, _ = _accum_with(ctx, 1, scene, opts, env)
            assert np.array_equal(a, d), sort
            assert rd == ra
        # The shade kernel at 4 blocks per SM (fewer registers): same image.
        ctx.set_shade_blocks(4)
        e, re_, _ = _accum_with(ctx, 1, scene, opts, env)
        assert np.array_equal(a, e) and re_ == ra
    finally:
        ctx.set_node_width(4, 4)
        ctx.set_material_sort(True)
        ctx.set_shade_blocks(3)
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)


def test_sync_resets_only_on_radiance_changes(ctx):
    scene = ts.area_light_scene(0.5, 0.0)
    o = ts.pt_opts(6, 8, 2)
    t = api.PathTracer(ctx)
    assert t.sync(scene, o)
    t.refine(2)
    display = o.replace(exposure=2.0, tone_map=ToneMap.AcesFitted,
                        path_trace=PathTraceOptions(samples_per_pixel=1000, max_bounces=2))
    assert not t.sync(scene, display)
    assert t.samples() == 2
    assert not t.is_converged()
    moved = display.replace(scene_camera=None, projection=Projection.Orthographic)
    assert t.sync(scene, moved)
    assert t.samples() == 0
    t.invalidate_scene()
    t.refine(1)
    assert t.sync(scene, moved)


def test_primary_misses_keep_background_bytes(ctx):
    scene = ts.area_light_scene(0.5, 0.0)
    o = ts.pt_opts(16, 4, 1, background=BackgroundColor((200, 10, 77, 128)), scene_camera=None,
                   camera=CameraSpec(0.0, 0.0, 3.0))
    img = api.PathTraceCudaRenderer(ctx).render(scene, o)
    assert tuple(img[0, 0]) == (200, 10, 77, 128)
    empty = api.PathTraceCudaRenderer(ctx).render(PreparedScene(), o)
    assert np.all(empty == np.array([200, 10, 77, 128], np.uint8))


def test_hostile_inputs_render_well_formed_images(ctx):
    # 1x1 renders, a degenerate triangle, huge coordinates, a scene of one
    # triangle; every render terminates with finite bytes.
    s = PreparedScene()
    m = s.add_material(ts.diffuse_material((0.5, 0.5, 0.5), 1.0))
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    s.add_primitive(Primitive(tri, np.array([0, 1, 2], np.uint32), material=m))
    s.add_primitive(Primitive(np.zeros((3, 3), np.float32), np.array([0, 1, 2], np.uint32), material=m))
    s.add_primitive(Primitive(tri * 1e30, np.array([0, 1, 2], np.uint32), material=m))
    for w, h in [(1, 1), (7, 3)]:
        o = ts.pt_opts(w, 4, 3, h=h, scene_camera=None)
        img = api.PathTraceCudaRenderer(ctx).render(s, o)
        assert img.shape == (h, w, 4)
        hdr = api.PathTraceCudaRenderer(ctx).render_hdr(s, o)
        assert np.all(np.isfinite(hdr))


def test_invalid_options_are_rejected(ctx):
    scene = ts.lambert_plane(0.5)
    t = api.PathTracer(ctx)
    with pytest.raises(api.RenderError) as e:
        t.sync(scene, ts.pt_opts(4, 1, 2000))
    assert e.value.status == abi.PT_ERR_INVALID_ARG


def test_make_renderer_arm(ctx):
    r = api.make_renderer(RenderBackend.PathTraceCuda, ctx)
    img = r.render(ts.lambert_plane(0.5), ts.pt_opts(8, 2, 1, ambient=1.0))
    assert img.shape == (8, 8, 4)
    with pytest.raises(NotImplementedError):
        api.make_renderer(RenderBackend.Scanline, ctx)


def test_scene_release_and_counts(ctx):
    scene, opts = ts.cornell_c0()
    desc = scene.to_desc(opts)
    sid = ctx.upload(desc)
    assert ctx.scene_bytes(sid) > 0
    st = ctx.bvh_stats(sid)
    assert st["max_depth"] < 64 and st["nodes"] >= 1
    ctx.release(sid)
    with pytest.raises(api.RenderError):
        ctx.release(sid)


def test_a_fresh_context_runs_the_wavefront_by_default():
    # The drop-in path (make_renderer / pt_create with nothing set) must run
    # the wavefront schedule, and its accumulator must equal the megakernel's.
    scene, opts = ts.sphere_grid_c1(64, 4)
    fresh = api.Context(0)
    try:
        fresh.set_stage_timing(True)  # only records per-stage device times
        t = api.PathTracer(fresh)
        t.sync(scene, opts)
        t.refine(4)
        stages = t.stage_ms()
        assert stages["extend"] > 0.0 and stages["shade"] > 0.0 and stages["shadow"] > 0.0, stages
        assert stages["megakernel"] == 0.0, stages
        wf = t.accum()
        t.close()
    finally:
        fresh.close()
    mk = api.Context(0)
    try:
        mk.set_schedule(abi.PT_SCHEDULE_MEGAKERNEL)
        t = api.PathTracer(mk)
        t.sync(scene, opts)
        t.refine(4)
        assert np.array_equal(t.accum(), wf)
        t.close()
    finally:
        mk.close()


def test_injected_allocation_failure_leaves_the_context_usable():
    # pt_debug_fail_allocations: host-side, no CUDA call fails. The sync
    # that needed an accumulator returns PT_ERR_OOM; the next one works and
    # renders what a fresh context renders.
    scene, opts = ts.cornell_c0()
    o = opts.replace(width=40, height=24, path_trace=PathTraceOptions(samples_per_pixel=4, max_bounces=4))
    c = api.Context(0)
    try:
        t = api.PathTracer(c)
        c.fail_allocations(1)
        with pytest.raises(api.RenderError) as ei:
            t.sync(scene, o)
        assert ei.value.status == abi.PT_ERR_OOM
        t.invalidate_scene()
        t.sync(scene, o)
        t.refine(4)
        got = t.accum()
        t.close()
        c.fail_allocations(1)  # a scene upload
        with pytest.raises(api.RenderError) as ei:
            c.upload(scene.to_desc(o))
        assert ei.value.status == abi.PT_ERR_OOM
    finally:
        c.close()
    fresh = api.Context(0)
    try:
        want = api.PathTracer(fresh)
        want.sync(scene, o)
        want.refine(4)
        assert np.array_equal(got, want.accum())
        want.close()
    finally:
        fresh.close()
