"""The oracle's RenderBackend::Raycast ShadingMode::Pbr, pinned to the
reference's own Pbr tests (tests/raycast_pbr.rs:101-690): emissive radiance
kept in HDR, ray-traced hard shadows for directional and point lights with
no acne or self-shadowing, MASK cut-outs and BLEND layers filtering shadow
rays, MASK / BLEND composited per camera ray, back-face culling, mirror
reflection fading with roughness and stopping at the cut-off, Fresnel-only
dielectric reflection, a glass ball lens inverting the background (and a
thin-walled ball not), Beer-Lambert tinting, an index-matched thin wall
being invisible, termination between parallel mirrors at any depth, and
determinism. Scanline-backend comparisons of the reference tests are left
out (that backend is not part of this library)."""
import math

import numpy as np

import raycast_pbr_scenes as P
from oxideav_render_b200 import abi, testscenes as ts
from oxideav_render_b200.options import BackgroundColor, LightSpec
from oxideav_render_b200.scene import Material, MaterialExt, Volume


def ray(oracle, scene, o):
    return oracle.raycast(scene, o)[1]


def test_hdr_output_keeps_radiance(oracle):
    # tests/raycast_pbr.rs:101-132.
    e = Material(base_color=(0.0, 0.0, 0.0, 1.0), emissive_factor=(1.0, 0.25, 0.0),
                 ext=MaterialExt(emissive_strength=4.0))
    scene = P.single_quad(e)
    o = P.opts(32, 32, ambient=0.0, use_scene_lights=False, light=LightSpec(intensity=0.0))
    hdr, img = oracle.raycast(scene, o)
    p = hdr[16, 16]
    assert abs(p[0] - 4.0) < 1e-3 and abs(p[1] - 1.0) < 1e-3, p
    assert tuple(img[0, 0]) == P.BG
    assert tuple(img[16, 16]) == (255, 255, 0, 255)


def test_ray_traced_shadows(oracle):
    # tests/raycast_pbr.rs:212-239 (the shadow-map comparison left out).
    scene = ts.shadow_box()
    off = P.opts(160, 120)
    on = off.replace(shadows=True)
    r_off, r_on = ray(oracle, scene, off), ray(oracle, scene, on)
    shadowed = P.project(scene, off, [0.0, 0.0, 0.45])
    lit = P.project(scene, off, [2.0, 0.0, 2.0])
    assert P.luma(P.px(r_on, shadowed)) + 40.0 < P.luma(P.px(r_off, shadowed))
    assert np.array_equal(P.px(r_on, lit), P.px(r_off, lit)), "no acne on the lit floor"
    top = P.project(scene, off, [0.0, 2.0, 0.0])
    assert np.array_equal(P.px(r_on, top), P.px(r_off, top)), "no self-shadowing"


def test_point_lights_cast_ray_traced_shadows(oracle):
    # tests/raycast_pbr.rs:241-265.
    scene = ts.cornell_box()
    off = P.opts(160, 120)
    a, b = ray(oracle, scene, off), ray(oracle, scene, off.replace(shadows=True))
    hidden = P.project(scene, off, [-0.9, -1.0, -0.9])
    lit = P.project(scene, off, [0.9, -1.0, -0.6])
    assert P.luma(P.px(b, hidden)) + 15.0 < P.luma(P.px(a, hidden))
    assert np.array_equal(P.px(b, lit), P.px(a, lit))


def test_mask_cutouts_and_blend_surfaces_filter_shadow_rays(oracle):
    # tests/raycast_pbr.rs:289-355.
    o = P.opts(160, 120, shadows=True)
    free = ray(oracle, P.occluder_scene(Material()), o.replace(shadows=False))
    mask_scene = P.occluder_scene(Material(), mask_texture=True)
    masked = ray(oracle, mask_scene, o)
    lit = dark = 0
    for c in ([-0.5, 0.0, -0.5], [0.5, 0.0, -0.5], [-0.5, 0.0, 0.5], [0.5, 0.0, 0.5]):
        xy = P.project(mask_scene, o, c)
        l, f = P.luma(P.px(masked, xy)), P.luma(P.px(free, xy))
        if abs(l - f) < 1.0:
            lit += 1
        elif l + 40.0 < f:
            dark += 1
    assert (lit, dark) == (2, 2), "two cut-out cells pass light"
    blend_scene = P.occluder_scene(Material(base_color=(1.0, 1.0, 1.0, 0.5), alpha_mode=abi.PT_ALPHA_BLEND))
    blended = ray(oracle, blend_scene, o)
    xy = P.project(blend_scene, o, [0.0, 0.0, 0.0])
    opaque = ray(oracle, P.occluder_scene(Material()), o)
    lb, lf, lo = P.luma(P.px(blended, xy)), P.luma(P.px(free, xy)), P.luma(P.px(opaque, xy))
    assert lo + 20.0 < lb and lb + 20.0 < lf, (lo, lb, lf)


def test_alpha_mask_and_blend_composite(oracle):
    # tests/raycast_pbr.rs:358-390.
    scene = ts.alpha_planes()
    o = P.opts(320, 240)
    img = ray(oracle, scene, o)

    def at(x, y):
        return P.px(img, P.project(scene, o, [x, y, 0.0])).astype(int)

    assert np.all(np.abs(at(-0.5, 0.5) - [188, 188, 0, 255]) <= 2), at(-0.5, 0.5)
    assert np.all(np.abs(at(-0.5, -0.5) - [188, 0, 188, 255]) <= 2), at(-0.5, -0.5)
    assert list(at(0.5, 0.5)) == [0, 0, 255, 255], "masked-out cell shows blue"
    assert list(at(0.5, -0.5)) == [0, 255, 0, 255], "masked-in cell green"
    lone = P.single_quad(P.unlit((1.0, 0.0, 0.0), 0.5, abi.PT_ALPHA_BLEND))
    img = ray(oracle, lone, P.opts(32, 32, background=BackgroundColor((0, 0, 255, 255))))
    assert tuple(img[16, 16]) == (188, 0, 188, 255)


def test_back_faces_culled_unless_double_sided(oracle):
    # tests/raycast_pbr.rs:393-407.
    m = P.unlit((1.0, 1.0, 1.0))
    scene = P.single_quad(m, P.rotate_y(math.pi))
    assert tuple(ray(oracle, scene, P.opts(16, 16))[8, 8]) == P.BG
    m2 = P.unlit((1.0, 1.0, 1.0))
    m2.double_sided = True
    assert tuple(ray(oracle, P.single_quad(m2, P.rotate_y(math.pi)), P.opts(16, 16))[8, 8]) != P.BG


def test_smooth_metal_mirrors_the_wall(oracle):
    # tests/raycast_pbr.rs:448-466.
    o = P.opts(128, 96)
    scene = P.mirror_scene(P.metal(0.0))
    xy = P.project(scene, o, [0.0, 0.0, -1.0])
    p = P.px(ray(oracle, scene, o), xy)
    assert p[0] > 240 and p[1] < 60 and p[2] < 60, p
    q = P.px(ray(oracle, scene, o.replace(max_ray_depth=0)), xy)
    assert q[0] < 200, q


def test_reflection_fades_with_roughness_and_stops_at_the_cutoff(oracle):
    # tests/raycast_pbr.rs:469-509 (the scanline comparison left out).
    o = P.opts(96, 72)

    def redness(r):
        scene = P.mirror_scene(P.metal(r))
        p = P.px(ray(oracle, scene, o), P.project(scene, o, [0.0, 0.0, -1.0])).astype(int)
        return p[0] - p[1]

    r0, r2, r4 = redness(0.0), redness(0.2), redness(0.4)
    assert r0 > r2 > r4, (r0, r2, r4)
    scene = P.mirror_scene(P.metal(0.6))
    assert np.array_equal(ray(oracle, scene, o), ray(oracle, scene, o.replace(max_ray_depth=0)))
    scene = P.mirror_scene(P.metal(0.0))
    assert np.array_equal(ray(oracle, scene, o.replace(reflection_roughness_cutoff=0.0)),
                          ray(oracle, scene, o.replace(max_ray_depth=0)))


def test_dielectric_mirror_reflects_by_fresnel_only(oracle):
    # tests/raycast_pbr.rs:512-529.
    o = P.opts(96, 72)
    glossy = ts.diffuse_material((0.05, 0.05, 0.05), 0.0)
    glossy.metallic = 0.0
    scene = P.mirror_scene(glossy)
    xy = P.project(scene, o, [0.0, 0.0, -1.0])
    pd = P.px(ray(oracle, scene, o), xy).astype(int)
    pm = P.px(ray(oracle, P.mirror_scene(P.metal(0.0)), o), xy).astype(int)
    assert pd[0] > pd[1] + 20, pd
    assert pd[0] < pm[0], (pd, pm)


def test_glass_sphere_inverts_the_background(oracle):
    # tests/raycast_pbr.rs:577-607.
    o = P.opts(128, 128, ambient=0.0)
    solid = P.lens_scene(P.glass(2.0))
    img = ray(oracle, solid, o)
    left = P.px(img, P.project(solid, o, [-0.4, 0.0, 0.9])).astype(int)
    right = P.px(img, P.project(solid, o, [0.4, 0.0, 0.9])).astype(int)
    assert left[1] > 2 * max(left[0], 10), left
    assert right[0] > 2 * max(right[1], 10), right
    thin = P.lens_scene(P.glass(0.0))
    left = P.px(ray(oracle, thin, o), P.project(thin, o, [-0.4, 0.0, 0.9])).astype(int)
    assert left[0] > 2 * max(left[1], 10), left
    c = P.px(ray(oracle, solid, o.replace(max_ray_depth=0)), P.project(solid, o, [0.0, 0.0, 1.0]))
    assert c[0] == c[1] == c[2], c


def test_volume_attenuation_tints_and_ior_one_is_invisible(oracle):
    # tests/raycast_pbr.rs:610-647.
    o = P.opts(96, 96, ambient=0.0)
    clear = P.lens_scene(P.glass(2.0))
    tinted = P.lens_scene(P.glass(2.0, attenuation_distance=0.5, attenuation_color=(0.2, 0.2, 1.0)))
    xy = P.project(clear, o, [-0.4, 0.0, 0.9])
    a, b = P.px(ray(oracle, clear, o), xy).astype(int), P.px(ray(oracle, tinted, o), xy).astype(int)
    assert b[1] + 60 < a[1], (a, b)
    o = o.replace(use_scene_lights=False, light=LightSpec(intensity=0.0))
    g = ray(oracle, P.lens_scene(P.glass(0.0, ior=1.0)), o)
    n = ray(oracle, P.lens_scene(None), o)
    assert ts.mean_abs_error(g, n) < 0.5


def test_deep_recursion_terminates_between_parallel_mirrors(oracle):
    # tests/raycast_pbr.rs:650-675.
    scene = P.parallel_mirrors()
    for depth in (0, 4, 16, 1000):
        img = ray(oracle, scene, P.opts(32, 32, max_ray_depth=depth, shadows=True))
        assert img.shape == (32, 32, 4)


def test_deterministic_with_aa_and_shadows(oracle):
    # tests/raycast_pbr.rs:678-689.
    scene = ts.cornell_box()
    o = P.opts(150, 101, shadows=True, aa=2)
    a, b = oracle.raycast(scene, o), oracle.raycast(scene, o)
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)) and np.array_equal(a[1], b[1])


def test_blend_layers_stop_at_the_layer_cap(oracle):
    # MAX_LAYERS (src/raycast.rs:126): 70 stacked BLEND planes render, and
    # the pixel behind all of them differs from a 60-plane stack.
    o = P.opts(24, 24)
    deep = oracle.raycast(P.blend_stack(70), o)[0]
    shallow = oracle.raycast(P.blend_stack(60), o)[0]
    assert np.all(np.isfinite(deep)) and not np.array_equal(deep, shallow)


# ---- the glTF BRDF, src/brdf.rs:150-211 ------------------------------------

def test_ggx_integrates_to_one_over_projected_hemisphere(oracle):
    for alpha in (0.1, 0.5, 1.0):
        n = 4000
        th = (np.arange(n) + 0.5) / n * (math.pi / 2)
        c = np.cos(th).astype(np.float32)
        d = np.array([oracle.gltf_d_ggx(float(x), alpha) for x in c], np.float64)
        total = float(np.sum(d * c.astype(np.float64) * np.sin(th) * 2.0 * math.pi * (math.pi / 2 / n)))
        assert abs(total - 1.0) < 0.02, (alpha, total)


def test_white_furnace_lambert_bound(oracle):
    steps = 200
    total = 0.0
    for i in range(steps):
        th = (i + 0.5) / steps * (math.pi / 2)
        for j in range(0, steps, 4):  # the integrand does not depend on phi
            ph = (j + 0.5) / steps * 2.0 * math.pi
            l = (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th))
            dw = math.sin(th) * (math.pi / 2 / steps) * (2.0 * math.pi / steps)
            total += oracle.gltf_brdf((1.0, 1.0, 1.0), 0.0, 1.0, 0.04, (0, 0, 1), (0, 0, 1), l)[1][0] * dw * 4
    assert 0.8 < total <= 1.02, total


def test_metals_have_no_diffuse_and_tinted_f0(oracle):
    (c_diff, f0, _), _ = oracle.gltf_brdf((1.0, 0.5, 0.0), 1.0, 0.5, 0.04, (0, 0, 1), (0, 0, 1), (0, 0, 1))
    assert c_diff == (0.0, 0.0, 0.0) and f0 == (1.0, 0.5, 0.0)
    assert oracle.gltf_schlick((0.04, 0.04, 0.04), 0.0) == (1.0, 1.0, 1.0)


def test_below_horizon_is_black(oracle):
    _, e = oracle.gltf_brdf((1.0, 1.0, 1.0), 0.0, 0.5, 0.04, (0, 0, 1), (0, 0, 1), (0, 0, -1))
    assert e == (0.0, 0.0, 0.0)
