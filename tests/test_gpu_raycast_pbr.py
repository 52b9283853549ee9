"""RenderBackend::Raycast ShadingMode::Pbr on the device (pt_raycast_render)
against the oracle's restatement of src/raycast.rs:518-768: HDR and RGBA8
bit-identical on scenes whose arithmetic is +, -, *, /, sqrt (directional,
point and spot lights, hard shadows through MASK / BLEND / transmissive
occluders, mirrors, thin walls, clear volumes, BLEND stacks past MAX_LAYERS,
16-bounce mirror recursion that needs the deep frame stacks, SSAA,
orthographic cameras, a device-built BVH); within 2e-5 relative where the
math library enters (logf / expf of Beer-Lambert absorption, log2f of
texture LOD from ray differentials and cones), since the device's and
glibc's f32 transcendental functions may round differently."""
import numpy as np
import pytest

import raycast_pbr_scenes as P
from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import BackgroundColor, CameraSpec, Projection, ToneMap
from oxideav_render_b200.scene import Material, MaterialExt, Transmission, spot_light

pytestmark = pytest.mark.gpu


def exact_case(name):
    bg = BackgroundColor((30, 60, 90, 255))
    if name == "cornell":
        return ts.cornell_box(), P.opts(64, 48, background=bg)
    if name == "cornell_shadows_aa":
        return ts.cornell_box(), P.opts(48, 40, shadows=True, aa=2)
    if name == "shadow_box":
        return ts.shadow_box(), P.opts(64, 48, shadows=True)
    if name == "alpha_planes":
        return ts.alpha_planes(), P.opts(64, 48, background=BackgroundColor((10, 20, 200, 128)))
    if name == "mask_occluder":
        return P.occluder_scene(Material(), mask_texture=True), P.opts(64, 48, shadows=True)
    if name == "blend_occluder":
        return (P.occluder_scene(Material(base_color=(1.0, 0.8, 0.6, 0.5), alpha_mode=abi.PT_ALPHA_BLEND)),
                P.opts(64, 48, shadows=True))
    if name == "tinted_pane_shadow":
        pane = Material(base_color=(0.9, 0.5, 0.2, 1.0), metallic=0.2, roughness=0.3,
                        ext=MaterialExt(transmission=Transmission(0.8)), double_sided=True)
        return P.occluder_scene(pane), P.opts(64, 48, shadows=True)
    if name == "mirror":
        return P.mirror_scene(P.metal(0.0)), P.opts(64, 48, shadows=True)
    if name == "rough_mirror":
        return P.mirror_scene(P.metal(0.2)), P.opts(64, 48)
    if name == "dielectric":
        glossy = ts.diffuse_material((0.05, 0.05, 0.05), 0.0)
        glossy.metallic = 0.0
        return P.mirror_scene(glossy), P.opts(64, 48)
    if name == "clear_ball":
        return P.lens_scene(P.glass(2.0), 32, 16), P.opts(48, 48, ambient=0.0)
    if name == "thin_ball":
        return P.lens_scene(P.glass(0.0), 32, 16), P.opts(48, 48)
    if name == "mirrors16":
        # Tinted facing mirrors with a lit block between them: 16 bounces
        # need the deep frame stacks.
        s = P.parallel_mirrors()
        s.materials[0].base_color = (0.95, 0.9, 0.8, 1.0)
        P.add(s, ts.cuboid([-0.1, -0.1, -0.6], [0.1, 0.1, -0.4]), ts.diffuse_material((0.8, 0.3, 0.2), 1.0))
        s.add_light(ts.point_light((1.0, 1.0, 1.0), 3.0), [0.5, 1.5, 0.0], [0.0, -1.0, 0.0])
        return s, P.opts(32, 32, max_ray_depth=16, shadows=True)
    if name == "blend_stack70":
        # About 3400 samples cross all 70 layers: more than the deep pass's
        # 2048 slots, so its threads take several samples each.
        return P.blend_stack(70), P.opts(64, 64, shadows=True)
    if name == "spheres":
        return ts.sphere_grid(3, 3, 24, 12), P.opts(64, 64, shadows=True, aa=2)
    if name == "ortho":
        s = ts.cornell_box()
        return s, P.opts(40, 40, scene_camera=None, projection=Projection.Orthographic,
                         camera=CameraSpec(20.0, 30.0, 1.0), shadows=True)
    if name == "backface":
        m = P.unlit((1.0, 1.0, 1.0))
        m.double_sided = True
        return P.single_quad(m, P.rotate_y(3.0)), P.opts(24, 24)
    if name == "spot":
        s = ts.shadow_box()
        s.add_light(spot_light((1.0, 0.9, 0.8), 30.0, 8.0, 0.15, 0.45), [1.5, 3.0, 1.0], [-0.4, -1.0, -0.3])
        return s, P.opts(64, 48, shadows=True)
    if name == "soup":
        s = ts.random_soup(40000, seed=5)
        s.add_light(ts.point_light((1.0, 0.9, 0.8), 4.0), [0.5, 1.5, 0.5], [0.0, -1.0, 0.0])
        return s, P.opts(48, 40, shadows=True)
    raise KeyError(name)


def close_case(name):
    if name == "tinted_ball":
        return (P.lens_scene(P.glass(2.0, attenuation_distance=0.5, attenuation_color=(0.2, 0.2, 1.0)), 32, 16),
                P.opts(48, 48, ambient=0.0))
    if name == "checker_floor":
        s, o = ts.sphere_grid_c1(64, 1)
        return s, P.opts(64, 64, scene_camera=o.scene_camera, shadows=True)
    if name == "normal_map":
        return ts.normal_mapped_quad(1.0), P.opts(32, 32, shadows=True)
    if name == "materials":
        return ts.material_extensions(), P.opts(48, 40, scene_camera=None, shadows=True)
    raise KeyError(name)


def render(ctx, scene, o):
    r = api.RaycastCudaRenderer(ctx)
    return r.render_hdr(scene, o), r.render(scene, o)


@pytest.mark.parametrize("name", ["cornell", "cornell_shadows_aa", "shadow_box", "alpha_planes", "mask_occluder",
                                  "blend_occluder", "tinted_pane_shadow", "mirror", "rough_mirror", "dielectric",
                                  "clear_ball", "thin_ball", "mirrors16", "blend_stack70", "spheres", "ortho",
                                  "backface", "spot", "soup"])
def test_pbr_equals_the_oracle(ctx, oracle, name):
    scene, o = exact_case(name)
    want_hdr, want_img = oracle.raycast(scene, o)
    got_hdr, got_img = render(ctx, scene, o)
    assert np.any(want_img != want_img[0, 0]), "degenerate case"
    assert np.array_equal(got_hdr.view(np.uint32), want_hdr.view(np.uint32)), \
        float(np.nanmax(np.abs(got_hdr - want_hdr)))
    assert np.array_equal(got_img, want_img)


@pytest.mark.parametrize("name", ["tinted_ball", "checker_floor", "normal_map", "materials"])
def test_pbr_matches_the_oracle_where_math_functions_enter(ctx, oracle, name):
    scene, o = close_case(name)
    want_hdr, want_img = oracle.raycast(scene, o)
    got_hdr, got_img = render(ctx, scene, o)
    assert np.allclose(got_hdr, want_hdr, rtol=2e-5, atol=2e-6), float(np.max(np.abs(got_hdr - want_hdr)))
    assert int(np.max(np.abs(got_img.astype(int) - want_img.astype(int)))) <= 1
    # Only pixels whose rays meet logf / expf / log2f can differ.
    assert np.mean(np.all(got_hdr == want_hdr, axis=2)) > 0.5


def test_pbr_display_transform_and_determinism(ctx, oracle):
    scene, o = exact_case("spheres")
    for tm, exposure in ((ToneMap.AcesFitted, 1.5), (ToneMap.Reinhard, 0.5)):
        oo = o.replace(tone_map=tm, exposure=exposure)
        assert np.array_equal(render(ctx, scene, oo)[1], oracle.raycast(scene, oo)[1])
    a, b = render(ctx, scene, o), render(ctx, scene, o)
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)) and np.array_equal(a[1], b[1])


def test_pbr_on_every_bvh_builder(ctx, oracle):
    # Hits do not depend on the tree, and the shadow transmittance product
    # does not depend on the order occluders are reported in.
    scene, o = exact_case("soup")
    want = oracle.raycast(scene, o)[0]
    try:
        for builder in (abi.PT_BVH_BUILD_HOST, abi.PT_BVH_BUILD_DEVICE, abi.PT_BVH_BUILD_DEVICE_PLOC):
            ctx.set_bvh_builder(builder)
            got = render(ctx, scene, o)[0]
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), builder
    finally:
        ctx.set_bvh_builder(abi.PT_BVH_BUILD_AUTO)
