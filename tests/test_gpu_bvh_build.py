"""Device-built BVHs (pt_set_bvh_builder): a scene whose tree is built on the
GPU — by the level-by-level binned-SAH build or by clustering — renders the
same accumulator, bit for bit, as with the host-built tree (closest hit =
smallest t, ties to the lowest global id, so hits do not depend on the
tree), on both schedules and both node layouts; the trees respect the
traversal stacks' depth limit and are deterministic, and the device
binned-SAH build gives the host builder's tree."""
import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import PathTraceOptions
from oxideav_render_b200.scene import Primitive

pytestmark = pytest.mark.gpu


def with_cloud(scene, tris: int, seed: int, center, size: float):
    """`scene` plus `tris` small diffuse triangles in a cube around `center`
    (enough triangles for the device builder, inside the camera's view)."""
    rng = np.random.default_rng(seed)
    m = scene.add_material(ts.diffuse_material((0.6, 0.6, 0.6), 1.0))
    c = np.asarray(center, np.float32) + (rng.random((tris, 1, 3)) - 0.5) * size
    d = rng.normal(size=(tris, 3, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    pos = (c + d * rng.uniform(0.003, 0.03, (tris, 1, 1))).astype(np.float32).reshape(-1, 3)
    scene.add_primitive(Primitive(np.ascontiguousarray(pos), material=m))
    return scene


def case(name):
    if name == "spheres":
        return ts.sphere_grid_c1(64, 2) + (None,)
    if name == "soup":
        return ts.random_soup(30000, seed=11), ts.pt_opts(48, 2, 6), None
    if name == "materials":
        return ts.material_extensions(), ts.pt_opts(48, 2, 6), None
    if name == "env":
        env = ts.env_noise(64, 32, np.random.default_rng(4))
        return with_cloud(ts.area_light_scene(0.35, 0.5), 3000, 1, (0, 0, 0), 1.0), ts.pt_opts(40, 4, 4), env
    if name == "alpha":
        return with_cloud(ts.alpha_planes(), 2000, 2, (0, 0, -0.5), 1.5), ts.pt_opts(40, 4, 4), None
    if name == "dispersion":
        return ts.dispersive_sphere(1.0), ts.pt_opts(40, 4, 8), None
    raise KeyError(name)


def render(ctx, builder, scene, opts, env, schedule):
    ctx.set_bvh_builder(builder)
    ctx.set_schedule(schedule)
    try:
        t = api.PathTracer(ctx)
        if env is not None:
            t.set_environment(api.EnvironmentMap(env))
        t.sync(scene, opts)
        t.refine(opts.path_trace.samples_per_pixel)
        sid = t._scene_id
        out = t.accum(), t.ray_counts(), ctx.bvh_stats(sid), ctx.bvh_on_device(sid)
        t.close()
        return out
    finally:
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)
        ctx.set_schedule(abi.PT_SCHEDULE_WAVEFRONT)


@pytest.mark.parametrize("name", ["spheres", "soup", "materials", "env", "alpha", "dispersion"])
def test_device_tree_renders_identically(ctx, name):
    scene, opts, env = case(name)
    a, ra, sa, da = render(ctx, abi.PT_BVH_BUILD_HOST, scene, opts, env, 0)
    assert not da
    for builder in (abi.PT_BVH_BUILD_DEVICE, abi.PT_BVH_BUILD_DEVICE_PLOC):
        for schedule in (0, 1):
            b, rb, sb, db = render(ctx, builder, scene, opts, env, schedule)
            assert db, "scene not built on the device"
            assert np.array_equal(a, b), (name, builder, schedule)
            assert ra == rb
            assert 0 < sb["max_depth"] <= 56 and sb["nodes"] > 0 and sb["leaves"] > 0
            assert sb["build_seconds"] > 0.0 and sb["sah_cost"] > 0.0
        try:
            # The two-child layout of the device tree, for both ray kinds.
            ctx.set_node_width(2, 2)
            c, rc, _, _ = render(ctx, builder, scene, opts, env, 1)
            assert np.array_equal(a, c) and rc == ra
        finally:
            ctx.set_node_width(4, 4)


def test_builder_selection(ctx):
    # Tiny scenes stay on the host even when the device builder is asked for;
    # AUTO builds large scenes on the device.
    small, o = ts.cornell_c0()
    o = o.replace(width=16, height=16, path_trace=PathTraceOptions(samples_per_pixel=1, max_bounces=2))
    assert not render(ctx, abi.PT_BVH_BUILD_DEVICE, small, o, None, 1)[3]
    big = ts.random_soup(20000, seed=3)
    assert render(ctx, abi.PT_BVH_BUILD_AUTO, big, ts.pt_opts(8, 1, 2), None, 1)[3]
    assert not render(ctx, abi.PT_BVH_BUILD_AUTO, ts.random_soup(2000, seed=3), ts.pt_opts(8, 1, 2), None, 1)[3]
    with pytest.raises(api.RenderError) as ei:
        ctx.set_bvh_builder(7)
    assert ei.value.status == abi.PT_ERR_INVALID_ARG


def test_device_trees_are_deterministic(ctx):
    scene = ts.random_soup(50000, seed=5)
    desc = scene.to_desc(ts.pt_opts(8, 1, 1))
    try:
        for builder in (abi.PT_BVH_BUILD_DEVICE, abi.PT_BVH_BUILD_DEVICE_PLOC):
            ctx.set_bvh_builder(builder)
            stats = []
            for _ in range(2):
                sid = ctx.upload(desc)
                assert ctx.bvh_on_device(sid)
                st = ctx.bvh_stats(sid)
                stats.append((st["nodes"], st["leaves"], st["max_depth"], st["sah_cost"], ctx.scene_bytes(sid)))
                ctx.release(sid)
            assert stats[0] == stats[1], builder
    finally:
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)


@pytest.mark.parametrize("name", ["spheres", "soup"])
def test_device_sah_build_gives_the_host_tree(ctx, name):
    # Same split rule, same float arithmetic: the same nodes and leaves
    # (these scenes never fall back to median splits).
    scene, opts, _ = case(name)
    desc = scene.to_desc(opts)
    got = {}
    try:
        for builder in (abi.PT_BVH_BUILD_HOST, abi.PT_BVH_BUILD_DEVICE):
            ctx.set_bvh_builder(builder)
            sid = ctx.upload(desc)
            got[builder] = ctx.bvh_stats(sid)
            ctx.release(sid)
    finally:
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)
    h, d = got[abi.PT_BVH_BUILD_HOST], got[abi.PT_BVH_BUILD_DEVICE]
    assert (h["nodes"], h["leaves"], h["max_depth"]) == (d["nodes"], d["leaves"], d["max_depth"])
    assert abs(h["sah_cost"] - d["sah_cost"]) <= 1e-6 * h["sah_cost"]


def test_hostile_geometry_on_every_builder(ctx):
    # Triangles with NaN or huge coordinates, zero-area and duplicated
    # triangles among ordinary ones: every builder's tree gives the host
    # tree's accumulator, and no device build fails.
    rng = np.random.default_rng(21)
    s = with_cloud(ts.area_light_scene(0.35, 0.5), 3000, 4, (0, 0, 0), 1.0)
    m = s.add_material(ts.diffuse_material((0.5, 0.7, 0.3), 1.0))
    bad = (rng.random((40, 3, 3)) - 0.5).astype(np.float32)
    bad[:10, 0, 0] = np.nan                  # NaN corners
    bad[10:20] = bad[10:11, :1]              # zero-area (all corners equal)
    bad[20:30] *= 1e30                       # enormous
    bad[30:40] = bad[30]                     # identical triangles
    s.add_primitive(Primitive(np.ascontiguousarray(bad.reshape(-1, 3)), material=m))
    o = ts.pt_opts(32, 2, 3)
    a, ra, _, _ = render(ctx, abi.PT_BVH_BUILD_HOST, s, o, None, 1)
    for builder in (abi.PT_BVH_BUILD_DEVICE, abi.PT_BVH_BUILD_DEVICE_PLOC):
        b, rb, st, on_device = render(ctx, builder, s, o, None, 1)
        assert on_device and st["max_depth"] <= 56
        assert np.array_equal(a, b), builder
        assert rb == ra


@pytest.mark.parametrize("name", ["spheres", "soup", "env", "alpha"])
def test_spatial_split_tree_renders_identically(ctx, name):
    # The spatial-split tree (a triangle referenced from several leaves, with
    # clipped leaf bounds) gives the host tree's accumulator bit for bit, on
    # both schedules; on the soup it holds more records than triangles.
    scene, opts, env = case(name)
    a, ra, sa, _ = render(ctx, abi.PT_BVH_BUILD_HOST, scene, opts, env, 1)
    for schedule in (0, 1):
        b, rb, sb, db = render(ctx, abi.PT_BVH_BUILD_HOST_SPATIAL, scene, opts, env, schedule)
        assert not db
        assert np.array_equal(a, b), (name, schedule)
        assert ra == rb
        assert 0 < sb["max_depth"] <= 56
    if name == "soup":
        assert sb["nodes"] > sa["nodes"]
        assert sb["sah_cost"] < sa["sah_cost"]
