"""Frame sources over the PathTraceCuda renderer (src/source.rs tests
:222-313 with this backend): a rendered frame reaches the video plane with
pixels other than the background, and every frame of an animated source
equals a direct render of the scene at that frame's time."""
import numpy as np
import pytest

from oxideav_render_b200 import api, testscenes as ts
from oxideav_render_b200.options import BackgroundColor, CameraSpec
from oxideav_render_b200.scene import PreparedScene, Primitive
from oxideav_render_b200.source import AnimatedRenderSource, Eof, RenderSource

pytestmark = pytest.mark.gpu


def one_triangle(green: float = 0.3) -> PreparedScene:
    s = PreparedScene()
    m = s.add_material(ts.diffuse_material((0.8, green, 0.2), 1.0))
    tri = np.array([[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.0, 0.5, 0.0]], np.float32)
    s.add_primitive(Primitive(tri, np.array([0, 1, 2], np.uint32), material=m))
    return s


def opts(w=32, h=None):
    return ts.pt_opts(w, 4, 2, h=h, background=BackgroundColor((255, 255, 255, 255)), scene_camera=None,
                      camera=CameraSpec(0.0, 0.0, 3.0), ambient=1.0)


def test_rendered_frame_has_non_background_pixels(ctx):
    src = RenderSource(one_triangle(), api.PathTraceCudaRenderer(ctx), opts())
    f = src.next_frame()
    px = np.frombuffer(f.planes[0].data, np.uint8).reshape(32, 32, 4)
    assert f.planes[0].stride == 32 * 4
    assert np.any(np.any(px != 255, axis=2))
    with pytest.raises(Eof):
        src.next_frame()


def test_non_square_frames(ctx):
    src = RenderSource(one_triangle(), api.PathTraceCudaRenderer(ctx), opts(48, 24))
    f = src.next_frame()
    assert f.planes[0].stride == 48 * 4 and len(f.planes[0].data) == 48 * 24 * 4


def test_animated_frames_equal_direct_renders(ctx):
    o = opts(40, 24)
    # The colour animates (the orbit camera frames the scene's bounds, so a
    # moving lone triangle would look the same in every frame).
    src = AnimatedRenderSource(lambda t: one_triangle(0.3 + 0.4 * t), api.PathTraceCudaRenderer(ctx), o, frames=3,
                               fps=(2, 1))
    frames = []
    for k in range(3):
        f = src.next_frame()
        assert f.pts == k
        t = k / 2
        want = api.PathTraceCudaRenderer(ctx).render(one_triangle(0.3 + 0.4 * t), o.replace(time=t))
        got = np.frombuffer(f.planes[0].data, np.uint8).reshape(24, 40, 4)
        assert np.array_equal(got, want), k
        frames.append(got)
    assert not np.array_equal(frames[0], frames[2])
    with pytest.raises(Eof):
        src.next_frame()


def moving_soup(t: float, seed: int = 3, tris: int = 20000) -> PreparedScene:
    """A random soup whose triangles drift with time (the same draw items and
    triangle counts in every frame): the refit case."""
    import copy
    s = copy.deepcopy(ts.random_soup(tris, seed=seed))
    rng = np.random.default_rng(seed + 1)
    for it in s.items:
        pos = it.positions.reshape(-1, 3, 3)
        vel = rng.normal(size=(pos.shape[0], 1, 3)).astype(np.float32) * 0.05
        it.positions = np.ascontiguousarray((pos + vel * np.float32(t)).reshape(it.positions.shape).astype(np.float32))
    s._bounds = None
    return s


@pytest.mark.parametrize("builder", ["auto", "spatial"])
def test_refitted_frames_equal_fresh_builds(ctx, builder):
    # render_frame refits the resident scene's tree from frame to frame; each
    # frame must equal a fresh render (fresh upload and BVH build) of the
    # scene at that time, bit for bit.
    from oxideav_render_b200 import abi
    o = ts.pt_opts(48, 4, 4, scene_camera=0, ambient=0.1)
    ctx.set_bvh_builder(abi.PT_BVH_BUILD_HOST_SPATIAL if builder == "spatial" else abi.PT_BVH_BUILD_AUTO)
    try:
        r = api.PathTraceCudaRenderer(ctx)
        for k, t in enumerate([0.0, 0.5, 1.0, 3.0]):
            scene = moving_soup(t)
            got = r.render_frame(scene, o.replace(time=t))
            sid = r.tracer.scene_id
            secs = ctx.upload_seconds(sid)
            if k > 0:
                # The tracer kept its scene id: the frame was a refit, not an upload.
                assert sid == first_sid
                assert secs["device_bvh"] >= 0.0
            else:
                first_sid = sid
            want = api.PathTraceCudaRenderer(ctx).render(scene, o.replace(time=t))
            assert np.array_equal(got, want), (builder, t)
        r.tracer.close()
    finally:
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)


def test_refit_rejects_a_different_topology(ctx):
    o = ts.pt_opts(32, 2, 2, scene_camera=0, ambient=0.1)
    a = moving_soup(0.0, seed=1, tris=5000)
    sid = ctx.upload(a.to_desc(o))
    try:
        with pytest.raises(api.RenderError):
            ctx.refit(sid, ts.random_soup(5001, seed=1).to_desc(o))
        # A frame of the same topology (the same soup, moved) refits in place.
        ctx.refit(sid, moving_soup(0.7, seed=1, tris=5000).to_desc(o))
    finally:
        ctx.release(sid)
