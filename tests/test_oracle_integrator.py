"""Oracle pins for the integrator and the trace layer: ports of
src/pathtrace.rs:3361-3750 and src/trace.rs:1222-1308 (known answers:
white furnace L = Le / (1 - rho), MIS / light-only / BSDF-only agreement,
error decreasing with spp, Cornell colour bleeding, determinism and refine
additivity, background bytes, uniform environment, glass Fresnel +
Beer-Lambert, point light 4/pi and the firefly clamp)."""
import math

import numpy as np
import pytest

from oxideav_render_b200 import testscenes as ts
from oxideav_render_b200.options import CameraSpec, LightStrategy, BackgroundColor
from oxideav_render_b200.scene import Camera

STRATEGIES = [LightStrategy.Mis, LightStrategy.LightOnly, LightStrategy.BsdfOnly]


def tracer(oracle, scene, opts, env=None):
    desc = scene.to_desc(opts)
    sc = oracle.OracleScene(desc)
    cam = Camera.resolve(scene, opts, max(opts.width, 1), max(opts.height, 1))
    t = oracle.OracleTracer(sc, cam, opts, env)
    t._keep = desc
    return t


def hdr(oracle, scene, opts, env=None):
    t = tracer(oracle, scene, opts, env)
    t.refine(max(opts.path_trace.samples_per_pixel, 1))
    return t.hdr()


def mean_rgb(img):
    return img[..., :3].astype(np.float64).mean(axis=(0, 1))


def test_white_furnace_converges_to_analytic_radiance(oracle):
    scene = ts.furnace_scene(0.5, 1.0)
    for s in STRATEGIES:
        m = mean_rgb(hdr(oracle, scene, ts.pt_opts(8, 64, 64, strategy=s)))
        assert np.all(np.abs(m - 2.0) < 0.04), (s, m)


@pytest.mark.parametrize("rough,metal", [(1.0, 0.0), (0.35, 0.5)])
def test_mis_light_only_and_bsdf_only_agree(oracle, rough, metal):
    scene = ts.area_light_scene(rough, metal)
    means = [mean_rgb(hdr(oracle, scene, ts.pt_opts(12, 256, 1, strategy=s)))[1] for s in STRATEGIES]
    ref = means[0]
    assert ref > 0.05, means
    for m in means:
        assert abs(m - ref) < 0.03 * ref, (rough, means)


def test_error_decreases_with_sample_count(oracle):
    scene = ts.area_light_scene(0.5, 0.0)
    ref = hdr(oracle, scene, ts.pt_opts(10, 1024, 3))
    errs = []
    for spp in [4, 16, 64]:
        img = hdr(oracle, scene, ts.pt_opts(10, spp, 3, seed=99))
        errs.append(float(np.sqrt(np.mean((img.astype(np.float64) - ref) ** 2))))
    assert errs[1] < errs[0] * 0.8 and errs[2] < errs[1] * 0.8, errs


def test_cornell_box_red_wall_bleeds_onto_floor(oracle):
    scene = ts.cornell_box()

    def red_ratio(bounces):
        img = hdr(oracle, scene, ts.pt_opts(32, 64, bounces))
        avg = lambda x0: img[28:31, x0:x0 + 3, :3].astype(np.float64).sum(axis=(0, 1))  # noqa: E731
        l, r = avg(4), avg(25)
        return (l[0] / l[1]) / (r[0] / r[1])

    assert abs(red_ratio(1) - 1.0) < 0.05
    assert red_ratio(6) > 1.15


def test_renders_are_deterministic_and_refinement_is_additive(oracle):
    scene = ts.area_light_scene(0.5, 0.0)
    o = ts.pt_opts(9, 8, 4)
    a = hdr(oracle, scene, o)
    b = hdr(oracle, scene, o)
    assert np.array_equal(a, b)
    t = tracer(oracle, scene, o)
    t.refine(3)
    t.refine(5)
    assert t.samples == 8
    assert np.array_equal(t.hdr(), a), "refine(3)+refine(5) must equal refine(8)"
    assert not np.array_equal(hdr(oracle, scene, ts.pt_opts(9, 8, 4, seed=1)), a)


def test_primary_misses_keep_background_bytes(oracle):
    scene = ts.area_light_scene(0.5, 0.0)
    o = ts.pt_opts(16, 4, 1, background=BackgroundColor((200, 10, 77, 128)), scene_camera=None,
                   camera=CameraSpec(0.0, 0.0, 3.0))
    t = tracer(oracle, scene, o)
    t.refine(4)
    img = t.image()
    assert tuple(img[0, 0]) == (200, 10, 77, 128)
    empty = ts.PreparedScene() if hasattr(ts, "PreparedScene") else None
    from oxideav_render_b200.scene import PreparedScene
    e = tracer(oracle, PreparedScene(), o)
    e.refine(4)
    assert np.all(e.image() == np.array([200, 10, 77, 128], np.uint8))


def test_uniform_environment_lights_a_lambert_plane(oracle):
    scene = ts.lambert_plane(0.5)
    env = oracle.OracleEnv(np.ones((8, 16, 4), np.float32), 1.0)
    for s in STRATEGIES:
        m = mean_rgb(hdr(oracle, scene, ts.pt_opts(6, 64, 2, strategy=s), env))
        assert abs(m[0] - 0.5) < 0.02, (s, m)
    m = mean_rgb(hdr(oracle, scene, ts.pt_opts(6, 64, 2, ambient=1.0)))
    assert abs(m[0] - 0.5) < 0.02, m


def test_smooth_glass_transmits_with_fresnel_and_beer_lambert(oracle):
    thin = mean_rgb(hdr(oracle, ts.glass_scene(False), ts.pt_opts(4, 16, 8)))[0]
    vol = mean_rgb(hdr(oracle, ts.glass_scene(True), ts.pt_opts(4, 16, 8)))[0]
    assert abs(thin - 0.92) < 0.03, thin
    assert abs(vol - 0.46) < 0.03, vol


def test_point_lights_and_clamp(oracle):
    scene = ts.point_light_plane()
    l = mean_rgb(hdr(oracle, scene, ts.pt_opts(2, 4, 1)))[0]
    assert abs(l - 4.0 / math.pi) < 0.01, l
    c = mean_rgb(hdr(oracle, scene, ts.pt_opts(2, 4, 1, clamp=0.5)))[0]
    assert abs(c - 0.5) < 1e-3, c


# ----------------------------------------------------------------------------- trace layer


def test_hits_back_wall_and_maps_back_to_item(oracle):
    scene = ts.cornell_box()
    sc = oracle.OracleScene(scene.to_desc())
    C = oracle.C
    f = lambda *v: np.array(v, np.float32)  # noqa: E731
    o, d = f(0.0, 0.5, 0.9), f(0.0, 0.0, -1.0)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    g, t, front = C.c_uint32(), C.c_float(), C.c_int()
    bary = np.zeros(3, np.float32)
    assert sc.triangle_count > 10
    assert oracle.lib().oracle_closest_hit(sc.ptr, fp(o), fp(d), 0.0, math.inf, C.byref(g), C.byref(t), fp(bary),
                                           C.byref(front))
    assert abs(t.value - 1.9) < 1e-4 and front.value == 1
    pos, ng, sn = np.zeros(3, np.float32), np.zeros(3, np.float32), np.zeros(3, np.float32)
    oracle.lib().oracle_surface(sc.ptr, g.value, fp(bary), fp(pos), fp(ng), fp(sn))
    assert abs(pos[2] + 1.0) < 1e-5 and abs(ng[2] - 1.0) < 1e-5
    assert oracle.lib().oracle_occluded(sc.ptr, fp(o), fp(d), 0.0, 2.0)
    assert not oracle.lib().oracle_occluded(sc.ptr, fp(o), fp(d), 0.0, 1.5)


def test_material_reads_factors(oracle):
    scene = ts.cornell_box()
    sc = oracle.OracleScene(scene.to_desc())
    C = oracle.C
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    o, d = np.array([0.0, 0.5, 0.0], np.float32), np.array([-1.0, 0.0, 0.0], np.float32)
    g, t, front = C.c_uint32(), C.c_float(), C.c_int()
    bary = np.zeros(3, np.float32)
    assert oracle.lib().oracle_closest_hit(sc.ptr, fp(o), fp(d), 0.0, math.inf, C.byref(g), C.byref(t), fp(bary),
                                           C.byref(front))
    out = np.zeros(6, np.float32)
    oracle.lib().oracle_material_base(sc.ptr, g.value, fp(bary), fp(out))
    assert out[0] > 0.6 and out[1] < 0.1, out


def test_emissive_table_is_power_proportional(oracle):
    scene, _ = ts.cornell_c0()
    sc = oracle.OracleScene(scene.to_desc())
    C = oracle.C
    n = C.c_uint32()
    tris, pmf, cdf = C.POINTER(C.c_uint32)(), C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
    oracle.lib().oracle_emissive_table(sc.ptr, C.byref(n), C.byref(tris), C.byref(pmf), C.byref(cdf))
    assert n.value == 2  # the ceiling quad
    assert abs(pmf[0] - 0.5) < 1e-6 and cdf[1] == 1.0
