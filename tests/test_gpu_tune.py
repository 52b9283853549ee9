"""The autotuner: it measures candidate configurations on a scratch
accumulator, records the fastest per scene class, and a tuned refine (or a
tuned server) gives bit-identical images."""
import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import PathTraceOptions
from oxideav_render_b200.serve import RenderServer

pytestmark = pytest.mark.gpu


def test_autotune_records_a_class_choice_and_keeps_images(ctx):
    ctx.tune_reset()
    scene, opts = ts.cornell_c0()
    o = opts.replace(width=64, height=48, path_trace=PathTraceOptions(samples_per_pixel=6, max_bounces=6))
    ref = api.PathTracer(ctx)
    ref.sync(scene, o)
    ref.refine(6)
    want = ref.accum()
    t = api.PathTracer(ctx)
    t.sync(scene, o)
    t.refine(2)
    assert ctx.tune_lookup(t) is None
    choice = ctx.autotune(t, 2)
    assert choice["schedule"] in (0, 1)
    assert choice["node_width_extension"] in (2, 4) and choice["node_width_shadow"] in (2, 4)
    assert choice["material_sort"] in (0, 1) and choice["wave_slots"] > 0
    assert choice["shade_blocks_per_sm"] in (3, 4) and choice["wave_arenas"] in (2, 3)
    assert choice["traversal_threads"] in (128, 256) and choice["claim_chunk"] in (1, 2, 4)
    assert choice["samples_per_s"] > 0
    assert ctx.tune_lookup(t) == choice
    # The tracer's own accumulator was not touched; tuned refines continue it.
    assert t.samples() == 2
    t.refine(4)
    assert np.array_equal(t.accum(), want)
    # Another scene of the same class shares the choice; another class does not.
    other = ts.random_soup(3000, seed=9)
    u = api.PathTracer(ctx)
    u.sync(other, ts.pt_opts(16, 1, 2))
    assert ctx.tune_lookup(u) is None
    ctx.tune_reset()
    assert ctx.tune_lookup(t) is None
    for x in (ref, t, u):
        x.close()


def test_tuned_server_images_match_plain(ctx):
    scenes = [(ts.cornell_c0()[0], ts.cornell_c0()[1].replace(width=40, height=32)),
              (ts.random_soup(8000, seed=4), ts.pt_opts(40, 3, 4, h=24)),
              (ts.sphere_grid_c1(48, 2)[0], ts.sphere_grid_c1(48, 2)[1])]
    plain = []
    for s, o in scenes:
        t = api.PathTracer(ctx)
        t.sync(s, o)
        t.refine(o.path_trace.samples_per_pixel)
        plain.append(t.hdr())
        t.close()
    srv = RenderServer(ctx, autotune=True)
    try:
        keys = [srv.register(s, o) for s, o in scenes]
        tickets = [srv.submit(k, o) for k, (_, o) in zip(keys, scenes)]
        for t, want in zip(tickets, plain):
            img, _ = srv.wait(t)
            assert np.array_equal(img, want)
        st = srv.stats()
        assert st["tuned_classes"] >= 2 and st["failed"] == 0
        # A second request of a tuned class is not tuned again.
        t2 = srv.submit(keys[0], scenes[0][1])
        assert np.array_equal(srv.wait(t2)[0], plain[0])
        assert srv.stats()["tuned_classes"] == st["tuned_classes"]
    finally:
        srv.close()


def test_server_without_material_sort_matches(ctx):
    s, o = ts.cornell_c0()
    o = o.replace(width=32, height=24, path_trace=PathTraceOptions(samples_per_pixel=3, max_bounces=5))
    t = api.PathTracer(ctx)
    t.sync(s, o)
    t.refine(3)
    want = t.hdr()
    t.close()
    srv = RenderServer(ctx, material_sort=False)
    try:
        k = srv.register(s, o)
        assert np.array_equal(srv.wait(srv.submit(k, o))[0], want)
    finally:
        srv.close()


@pytest.mark.parametrize("threads,chunk", [(128, 1), (256, 2), (256, 4), (128, 4)])
def test_traversal_block_size_and_claim_chunk_keep_images(ctx, threads, chunk):
    # The traversal kernels' block size and refill chunk only change which
    # lane traces which ray and when: accumulators and ray counts are equal.
    cases = [(ts.random_soup(20000, seed=3), ts.pt_opts(48, 4, 6)), ts.sphere_grid_c1(48, 2)]
    for scene, o in cases:
        ref = api.PathTracer(ctx)
        ref.sync(scene, o)
        ref.refine(o.path_trace.samples_per_pixel)
        want, rays = ref.accum(), ref.ray_counts()
        ref.close()
        ctx.set_traversal(threads, chunk)
        try:
            t = api.PathTracer(ctx)
            t.sync(scene, o)
            t.refine(o.path_trace.samples_per_pixel)
            assert np.array_equal(t.accum(), want)
            assert t.ray_counts() == rays
            t.close()
        finally:
            ctx.set_traversal(256, 1)
