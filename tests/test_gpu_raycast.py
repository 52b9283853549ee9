"""RenderBackend::Raycast on the device (pt_raycast_render) against the
oracle's restatement of src/raycast.rs: HDR and RGBA8 images bit-identical
for every legacy shading mode, with and without SSAA, on perspective and
orthographic cameras, scene cameras, textured / metallic / transmissive /
alpha-mode / large (device-BVH) scenes, deep Whitted recursion between two
mirrors, and the display transform's tone maps and exposure."""
import ctypes as C

import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import (BackgroundColor, CameraSpec, LightSpec, Projection, RenderBackend,
                                         RenderOptions, ShadingMode, ToneMap)
from oxideav_render_b200.scene import Material, PreparedScene, Primitive

pytestmark = pytest.mark.gpu

MODES = [ShadingMode.Flat, ShadingMode.Gouraud, ShadingMode.Phong, ShadingMode.Wireframe,
         ShadingMode.NormalDebug, ShadingMode.DepthDebug]


def mirrors():
    """Two facing mirrors with a diffuse ball of triangles between them."""
    s = PreparedScene()
    mirror = s.add_material(Material(base_color=(0.9, 0.95, 0.9, 1.0), metallic=1.0, roughness=0.0))
    for z in (-1.0, 1.0):
        p = np.array([[-2, -2, z], [2, -2, z], [-2, 2, z], [2, -2, z], [2, 2, z], [-2, 2, z]], np.float32)
        s.add_primitive(Primitive(p, np.arange(6, dtype=np.uint32), material=mirror))
    soup = ts.random_soup(300, seed=3)
    for it in soup.items[:1]:
        s.add_primitive(Primitive(np.ascontiguousarray(it.positions - 0.5), material=s.add_material(
            ts.diffuse_material((0.8, 0.4, 0.2), 1.0))))
    s.add_camera([0.3, 0.2, 0.9], [0.0, 0.0, -1.0], 1.0)
    return s


def case(name):
    bg = BackgroundColor((30, 60, 90, 255))
    if name == "cornell":
        s, o = ts.cornell_c0()
        return s, RenderOptions(width=48, height=48, scene_camera=o.scene_camera, background=bg)
    if name == "spheres":
        s, o = ts.sphere_grid_c1(40, 1)
        return s, RenderOptions(width=40, height=40, scene_camera=o.scene_camera, background=bg, max_ray_depth=3)
    if name == "materials":
        return ts.material_extensions(), RenderOptions(width=40, height=32, background=bg, max_ray_depth=4)
    if name == "alpha":
        return ts.alpha_planes(), RenderOptions(width=32, height=32, scene_camera=0, background=bg)
    if name == "soup":
        return ts.random_soup(40000, seed=5), RenderOptions(width=48, height=40, scene_camera=0, background=bg,
                                                           light=LightSpec(30.0, 60.0, 1.5))
    if name == "ortho":
        s, o = ts.cornell_c0()
        return s, RenderOptions(width=40, height=40, projection=Projection.Orthographic,
                                camera=CameraSpec(20.0, 30.0, 1.0), background=bg)
    if name == "mirrors":
        return mirrors(), RenderOptions(width=40, height=40, scene_camera=0, background=bg, max_ray_depth=16)
    raise KeyError(name)


def compare(ctx, oracle, scene, opts):
    r = api.RaycastCudaRenderer(ctx)
    want_hdr, want_img = oracle.raycast(scene, opts)
    got_hdr = r.render_hdr(scene, opts)
    got_img = r.render(scene, opts)
    assert np.array_equal(got_hdr.view(np.uint32), want_hdr.view(np.uint32)), \
        float(np.max(np.abs(got_hdr - want_hdr)))
    assert np.array_equal(got_img, want_img)
    return got_img


@pytest.mark.parametrize("name", ["cornell", "spheres", "materials", "alpha", "soup", "ortho", "mirrors"])
def test_device_raycast_equals_the_oracle(ctx, oracle, name):
    scene, opts = case(name)
    for mode in MODES:
        compare(ctx, oracle, scene, opts.replace(shading=mode))
    compare(ctx, oracle, scene, opts.replace(shading=ShadingMode.Phong, aa=2))


def test_display_transform_and_aa(ctx, oracle):
    scene, opts = case("spheres")
    for tm, exposure, aa in ((ToneMap.AcesFitted, 1.5, 1), (ToneMap.Reinhard, 0.5, 3), (ToneMap.Clamp, 4.0, 2)):
        compare(ctx, oracle, scene, opts.replace(tone_map=tm, exposure=exposure, aa=aa))
    # The debug views ignore exposure and tone mapping.
    a = compare(ctx, oracle, scene, opts.replace(shading=ShadingMode.NormalDebug, exposure=3.0,
                                                 tone_map=ToneMap.AcesFitted))
    b = compare(ctx, oracle, scene, opts.replace(shading=ShadingMode.NormalDebug))
    assert np.array_equal(a, b)


def test_backend_arm_and_errors(ctx):
    r = api.make_renderer(RenderBackend.Raycast, ctx)
    img = r.render(ts.lambert_plane(0.5), RenderOptions(width=8, height=6, background=BackgroundColor((1, 2, 3, 4))))
    assert img.shape == (6, 8, 4)
    pbr = r.render(ts.lambert_plane(0.5), RenderOptions(width=8, height=8, shading=ShadingMode.Pbr))
    assert pbr.shape == (8, 8, 4)
    bad = RenderOptions(width=8, height=8).to_raycast_c(0.01, 100.0)
    bad.aa = 9
    cam = abi.pt_camera()
    assert ctx.lib.pt_raycast_render(ctx.ptr, 0, C.byref(cam), C.byref(bad), None, 0, None, 0) == abi.PT_ERR_INVALID_ARG
    empty = r.render(PreparedScene(), RenderOptions(width=5, height=3, background=BackgroundColor((42, 7, 99, 255))))
    assert np.all(empty == np.array([42, 7, 99, 255], np.uint8))
