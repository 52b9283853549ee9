"""The render server: every served image is bit-identical to rendering the
request alone with a PathTracer (same scene, options, sample count), with
requests mixed in shared waves, arriving while others run, continued on
live accumulators, and with scenes evicted and re-admitted under an HBM
budget. Admission failures surface as request errors."""
import threading
import time

import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import PathTraceOptions
from oxideav_render_b200.serve import RenderServer

pytestmark = pytest.mark.gpu


def scenes_and_requests():
    rng = np.random.default_rng(5)
    c0, o0 = ts.cornell_c0()
    c1, o1 = ts.sphere_grid_c1(64, 2)
    soup = ts.random_soup(20000, seed=3)
    env = api.EnvironmentMap(ts.env_noise(32, 16, rng))
    area = ts.area_light_scene(0.35, 0.5)
    mats = ts.material_extensions()
    scenes = [(c0, o0, None), (c1, o1, None), (soup, ts.pt_opts(48, 1, 4), None), (area, ts.pt_opts(24, 1, 3), env),
              (mats, ts.pt_opts(40, 1, 6), None)]
    reqs = [  # (scene index, options)
        (0, o0.replace(width=48, height=40, path_trace=PathTraceOptions(samples_per_pixel=5, max_bounces=8))),
        (1, o1.replace(path_trace=PathTraceOptions(samples_per_pixel=3, max_bounces=4))),
        (2, ts.pt_opts(33, 7, 2, h=21)),
        (3, ts.pt_opts(24, 4, 3)),
        (4, ts.pt_opts(40, 2, 6)),
        (0, o0.replace(width=17, height=9, path_trace=PathTraceOptions(samples_per_pixel=9, max_bounces=2, seed=5))),
        (2, ts.pt_opts(64, 3, 8, h=64, seed=9)),
        (1, o1.replace(width=32, height=16, path_trace=PathTraceOptions(samples_per_pixel=1, max_bounces=2))),
    ]
    return scenes, reqs


def plain(ctx, scene, opts, env, extra=0):
    """The plain path: a PathTracer synced and refined alone (+ `extra`)."""
    t = api.PathTracer(ctx)
    if env is not None:
        t.set_environment(env)
    t.sync(scene, opts)
    t.refine(opts.path_trace.samples_per_pixel)
    first = t.hdr()
    if extra:
        t.refine(extra)
    out = (first, t.hdr())
    t.close()
    return out


@pytest.fixture(scope="module")
def workload(ctx):
    scenes, reqs = scenes_and_requests()
    ref = [plain(ctx, scenes[k][0], o, scenes[k][2], extra=4) for k, o in reqs]
    return scenes, reqs, ref


def register_all(srv, scenes):
    return [srv.register(s, o, e) for s, o, e in scenes]


@pytest.mark.parametrize("megakernel,overlap,slots", [(False, True, 0), (False, True, 20000), (False, False, 20000),
                                                      (True, False, 6000)])
def test_served_images_match_plain(ctx, workload, megakernel, overlap, slots):
    # Wavefront waves overlapped in two arenas (the default) or one at a
    # time, large or small waves, and the megakernel: images equal the
    # plain path's.
    scenes, reqs, ref = workload
    srv = RenderServer(ctx, wave_slots=slots, megakernel=megakernel, wave_overlap=overlap)
    try:
        keys = register_all(srv, scenes)
        tickets = [srv.submit(keys[k], o) for k, o in reqs]
        conts = [srv.submit_continuation(t, 4) for t in tickets]  # queued behind their base requests
        for i, t in enumerate(tickets):
            img, st = srv.wait(t)
            assert np.array_equal(img, ref[i][0]), f"request {i}"
            assert st["samples"] == reqs[i][1].path_trace.samples_per_pixel
            assert st["latency_ms"] >= st["queue_ms"] >= 0.0
        for i, t in enumerate(conts):
            img, st = srv.wait(t)
            assert np.array_equal(img, ref[i][1]), f"continuation {i}"
            assert st["samples"] == reqs[i][1].path_trace.samples_per_pixel + 4
        s = srv.stats()
        assert s["completed"] == 2 * len(reqs) and s["failed"] == 0
        assert s["waves"] >= 1 and s["rays"] > 0 and s["gpu_ms"] > 0.0
        for t in tickets + conts:
            srv.release(t)
    finally:
        srv.close()


def test_requests_from_many_threads(ctx, workload):
    """Requests arrive from several threads while others are on the GPU."""
    scenes, reqs, ref = workload
    srv = RenderServer(ctx, wave_slots=20000)
    keys = register_all(srv, scenes)
    results = {}
    errors = []

    def client(idx):
        try:
            for rep in range(3):
                i = (idx + rep) % len(reqs)
                t = srv.submit(keys[reqs[i][0]], reqs[i][1])
                img, _ = srv.wait(t)
                results[(idx, rep)] = (i, img)
                srv.release(t)
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    th = [threading.Thread(target=client, args=(k,)) for k in range(6)]
    for x in th:
        x.start()
    for x in th:
        x.join(timeout=300)
    srv.close()
    assert not errors, errors
    assert len(results) == 18
    for (i, img) in results.values():
        assert np.array_equal(img, ref[i][0])


def test_lru_eviction_under_budget(ctx, workload):
    scenes, reqs, ref = workload
    probe = RenderServer(ctx)
    keys = register_all(probe, scenes)
    sizes = [probe.scene_info(k)["device_bytes"] for k in keys]
    probe.close()
    # Room for the largest scene plus a little: most admissions evict.
    srv = RenderServer(ctx, hbm_budget_bytes=max(sizes) + 4096, max_active=1)
    try:
        keys = register_all(srv, scenes)
        order = list(range(len(reqs))) * 2
        tickets = [srv.submit(keys[reqs[i][0]], reqs[i][1]) for i in order]
        for i, t in zip(order, tickets):
            img, _ = srv.wait(t)
            assert np.array_equal(img, ref[i][0])
        s = srv.stats()
        assert s["scene_evictions"] > 0
        assert s["scene_uploads"] > len(scenes)
        assert s["peak_resident_bytes"] <= max(sizes) + 4096
        assert s["resident_scenes"] == 1
    finally:
        srv.close()


def test_scene_over_budget_fails_the_request(ctx):
    scene, opts = ts.cornell_c0()
    srv = RenderServer(ctx, hbm_budget_bytes=1024)
    try:
        key = srv.register(scene, opts)
        t = srv.submit(key, opts.replace(width=8, height=8))
        with pytest.raises(api.RenderError) as ei:
            srv.wait(t)
        assert ei.value.status == abi.PT_ERR_OOM
        # Its continuation inherits the failure.
        with pytest.raises(api.RenderError):
            srv.submit_continuation(t, 1)
        srv.release(t)
        assert srv.stats()["failed"] == 1
    finally:
        srv.close()


def test_ticket_and_scene_rules(ctx):
    scene, opts = ts.cornell_c0()
    small = opts.replace(width=16, height=16, path_trace=PathTraceOptions(samples_per_pixel=2, max_bounces=3))
    srv = RenderServer(ctx)
    try:
        key = srv.register(scene, small)
        t = srv.submit(key, small)
        img, st = srv.wait(t)
        assert img.shape == (16, 16, 4) and st["samples"] == 2
        # A finished request can be continued until it is released.
        c = srv.submit_continuation(t, 3)
        assert srv.wait(c)[1]["samples"] == 5
        srv.release(t)
        srv.release(c)
        with pytest.raises(api.RenderError) as ei:
            srv.submit_continuation(t, 1)
        assert ei.value.status == abi.PT_ERR_NOT_FOUND
        with pytest.raises(api.RenderError) as ei:
            srv.submit(key, small, samples=0)
        assert ei.value.status == abi.PT_ERR_INVALID_ARG
        # Released accumulations are freed by the worker.
        for _ in range(100):
            if srv.stats()["accumulators"] == 0:
                break
            time.sleep(0.01)
        assert srv.stats()["accumulators"] == 0
        srv.unregister(key)
        with pytest.raises(KeyError):
            srv.submit(key, small)
    finally:
        srv.close()


def test_destroy_with_queued_requests(ctx):
    """Closing a server with work queued cancels it cleanly."""
    scene, opts = ts.sphere_grid_c1(128, 64)
    srv = RenderServer(ctx, max_active=1)
    key = srv.register(scene, opts)
    for _ in range(4):
        srv.submit(key, opts)
    srv.close()


def _plain_hdr(ctx, scene, opts, spp=None):
    t = api.PathTracer(ctx)
    t.sync(scene, opts)
    t.refine(opts.path_trace.samples_per_pixel if spp is None else spp)
    out = t.hdr()
    t.close()
    return out


def _status_of(srv, ticket):
    with pytest.raises(api.RenderError) as ei:
        srv.wait(ticket)
    return ei.value.status


def test_cancel_a_queued_request(ctx):
    # One request at a time: the second one waits in the queue behind a long
    # first one and is cancelled there; its continuation fails with it; the
    # long one and a later request still equal the plain path.
    soup = ts.random_soup(20000, seed=3)
    big = ts.pt_opts(256, 64, 4)
    small = ts.pt_opts(32, 2, 3)
    srv = RenderServer(ctx, max_active=1, wave_slots=1 << 16)
    try:
        k = srv.register(soup, big)
        a = srv.submit(k, big)
        b = srv.submit(k, small)
        c = srv.submit_continuation(b, 2)
        srv.cancel(b)
        assert _status_of(srv, b) == abi.PT_ERR_CANCELLED
        assert _status_of(srv, c) in (abi.PT_ERR_CANCELLED, abi.PT_ERR_INVALID_ARG)
        img, _ = srv.wait(a)
        assert np.array_equal(img, _plain_hdr(ctx, soup, big))
        d = srv.submit(k, small)
        assert np.array_equal(srv.wait(d)[0], _plain_hdr(ctx, soup, small))
        s = srv.stats()
        assert s["cancelled"] == 1 and s["failed"] >= 2 and s["completed"] == 2
        for t in (a, b, c, d):
            srv.release(t)
        with pytest.raises(api.RenderError) as ei:
            srv.cancel(a)
        assert ei.value.status == abi.PT_ERR_NOT_FOUND
    finally:
        srv.close()


def test_cancel_a_running_request(ctx):
    # Small waves make the request span hundreds of waves; it is cancelled
    # while they run. Its accumulation can no longer be continued; the
    # server goes on serving.
    soup = ts.random_soup(20000, seed=3)
    big = ts.pt_opts(256, 256, 4)
    small = ts.pt_opts(32, 2, 3)
    srv = RenderServer(ctx, wave_slots=1 << 14)
    try:
        k = srv.register(soup, big)
        a = srv.submit(k, big)
        for _ in range(2000):
            if srv.stats()["waves"] >= 2:
                break
            time.sleep(0.001)
        assert srv.poll(a) is None  # still running
        srv.cancel(a)
        assert _status_of(srv, a) == abi.PT_ERR_CANCELLED
        with pytest.raises(api.RenderError):
            srv.submit_continuation(a, 1)
        with pytest.raises(api.RenderError) as ei:
            srv.cancel(a)
        assert ei.value.status == abi.PT_ERR_INVALID_ARG  # already finished
        e = srv.submit(k, small)
        assert np.array_equal(srv.wait(e)[0], _plain_hdr(ctx, soup, small))
        srv.release(a)
        srv.release(e)
        assert srv.stats()["cancelled"] == 1
    finally:
        srv.close()


def test_poll_bounded_wait_and_deadline(ctx):
    soup = ts.random_soup(20000, seed=3)
    big = ts.pt_opts(256, 64, 4)
    small = ts.pt_opts(32, 2, 3)
    srv = RenderServer(ctx, max_active=1, wave_slots=1 << 16)
    try:
        k = srv.register(soup, big)
        a = srv.submit(k, big)
        assert srv.poll(a) is None
        assert srv.poll_status(a) == abi.PT_ERR_NOT_READY
        assert srv.wait(a, timeout_ms=1) is None  # PT_ERR_TIMEOUT from the bounded wait
        rc = srv.lib.pt_server_wait(srv.ptr, a, 1, None, 0, None)
        assert rc in (abi.PT_ERR_TIMEOUT, abi.PT_OK)
        # Queued behind `a` with a 1 ms deadline: it times out.
        b = srv.submit(k, small, deadline_ms=1)
        assert _status_of(srv, b) == abi.PT_ERR_TIMEOUT
        img, _ = srv.wait(a)
        assert np.array_equal(img, _plain_hdr(ctx, soup, big))
        got = srv.poll(a)
        assert got is not None and np.array_equal(got[0], img)
        # A generous deadline does not fire.
        c = srv.submit(k, small, deadline_ms=600000)
        assert np.array_equal(srv.wait(c)[0], _plain_hdr(ctx, soup, small))
        s = srv.stats()
        assert s["timed_out"] == 1 and s["completed"] == 2
        for t in (a, b, c):
            srv.release(t)
    finally:
        srv.close()


def test_injected_allocation_failures_surface_as_oom(ctx):
    # Host-side injection: no CUDA call fails, the server's allocation
    # points report out of memory. The failed requests end with PT_ERR_OOM
    # and the server keeps serving.
    scene, opts = ts.cornell_c0()
    small = opts.replace(width=24, height=16, path_trace=PathTraceOptions(samples_per_pixel=3, max_bounces=4))
    want = _plain_hdr(ctx, scene, small)
    srv = RenderServer(ctx)
    try:
        k = srv.register(scene, small)
        srv.fail_allocations(1)  # the scene's first device commit
        a = srv.submit(k, small)
        assert _status_of(srv, a) == abi.PT_ERR_OOM
        assert not srv.scene_info(k)["resident"]
        b = srv.submit(k, small)
        assert np.array_equal(srv.wait(b)[0], want)
        srv.fail_allocations(1)  # the next request's accumulator
        c = srv.submit(k, small)
        assert _status_of(srv, c) == abi.PT_ERR_OOM
        d = srv.submit(k, small)
        assert np.array_equal(srv.wait(d)[0], want)
        s = srv.stats()
        assert s["failed"] == 2 and s["completed"] == 2
        for t in (a, b, c, d):
            srv.release(t)
    finally:
        srv.close()
