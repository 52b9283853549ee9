"""The oracle's RenderBackend::Raycast legacy shading modes, pinned to the
reference's own tests of src/raycast.rs (:823-1250): every mode paints the
triangle, an empty scene is pure background, output size with SSAA,
wireframe sparser than flat, Phong never brighter than the base colour on a
face lit off-axis, Whitted shadow rays, mirror reflection, refraction
through a transmissive pane, unlit and emissive materials, and the helper
identities (reflect / refract)."""
import numpy as np
import pytest

from oxideav_render_b200 import testscenes as ts
from oxideav_render_b200.options import (BackgroundColor, CameraSpec, LightSpec, RenderOptions, ShadingMode)
from oxideav_render_b200.scene import (Material, MaterialExt, PreparedScene, Primitive, Transmission)

WHITE = BackgroundColor((255, 255, 255, 255))
MODES = [ShadingMode.Flat, ShadingMode.Gouraud, ShadingMode.Phong, ShadingMode.Wireframe,
         ShadingMode.NormalDebug, ShadingMode.DepthDebug]


def unit_triangle(normals=None, material=None):
    s = PreparedScene()
    tri = np.array([[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.0, 0.5, 0.0]], np.float32)
    s.add_primitive(Primitive(tri, np.array([0, 1, 2], np.uint32), normals=normals, material=material))
    return s


def quad(y, half, normal_up=True, material=None):
    p = np.array([[-half, y, -half], [half, y, -half], [-half, y, half], [half, y, -half], [half, y, half],
                  [-half, y, half]], np.float32)
    n = np.tile(np.array([[0.0, 1.0 if normal_up else -1.0, 0.0]], np.float32), (6, 1)) if normal_up is not None \
        else None
    return Primitive(p, np.arange(6, dtype=np.uint32), normals=n, material=material)


def non_bg(img, bg):
    return int(np.sum(np.any(img != np.array(bg, np.uint8), axis=2)))


def test_every_mode_paints_the_triangle(oracle):
    for mode in MODES:
        _, img = oracle.raycast(unit_triangle(), RenderOptions(width=64, height=64, shading=mode, background=WHITE))
        assert non_bg(img, (255, 255, 255, 255)) > 0, mode


def test_empty_scene_yields_pure_background(oracle):
    _, img = oracle.raycast(PreparedScene(), RenderOptions(width=8, height=8,
                                                           background=BackgroundColor((42, 7, 99, 255))))
    assert np.all(img == np.array([42, 7, 99, 255], np.uint8))


def test_output_dimensions_with_and_without_aa(oracle):
    for aa in (1, 2, 4):
        hdr, img = oracle.raycast(unit_triangle(), RenderOptions(width=33, height=17, aa=aa, background=WHITE))
        assert img.shape == (17, 33, 4) and hdr.shape == (17, 33, 4)


def test_wireframe_paints_fewer_pixels_than_flat(oracle):
    o = RenderOptions(width=64, height=64, background=WHITE)
    _, flat = oracle.raycast(unit_triangle(), o.replace(shading=ShadingMode.Flat))
    _, wire = oracle.raycast(unit_triangle(), o.replace(shading=ShadingMode.Wireframe))
    bg = (255, 255, 255, 255)
    assert 0 < non_bg(wire, bg) < non_bg(flat, bg)


def test_phong_is_not_brighter_than_the_base_colour(oracle):
    scene = unit_triangle(normals=np.tile(np.array([[0.0, 0.0, 1.0]], np.float32), (3, 1)))
    _, img = oracle.raycast(scene, RenderOptions(width=32, height=32, shading=ShadingMode.Phong, background=WHITE))
    painted = img[np.any(img != 255, axis=2)]
    assert len(painted) > 0
    flat = np.array([219, 219, 225])  # linear (0.7, 0.7, 0.75) in sRGB bytes
    assert np.all(painted[:, :3] <= flat)


def test_shadow_ray_darkens_occluded_floor(oracle):
    bg = (255, 0, 255, 255)
    o = RenderOptions(width=48, height=48, shading=ShadingMode.Phong, background=BackgroundColor(bg),
                      light=LightSpec(0.0, 45.0, 1.0), camera=CameraSpec(80.0, 0.0, 1.5))
    scene = PreparedScene()
    scene.add_primitive(quad(0.0, 1.0))
    scene.add_primitive(quad(0.5, 0.3, normal_up=None))
    control = PreparedScene()
    control.add_primitive(quad(0.0, 1.0))

    def min_luma(img):
        px = img[np.any(img != np.array(bg, np.uint8), axis=2)]
        return int(px[:, 0].min()) if len(px) else 255

    assert min_luma(oracle.raycast(scene, o)[1]) <= 120
    assert min_luma(oracle.raycast(control, o)[1]) >= 160


def test_metallic_floor_reflects_a_red_wall(oracle):
    bg = (0, 0, 0, 255)
    o = RenderOptions(width=48, height=48, shading=ShadingMode.Phong, background=BackgroundColor(bg),
                      camera=CameraSpec(30.0, 0.0, 1.2), max_ray_depth=2)

    def scene(metal):
        s = PreparedScene()
        fm = s.add_material(Material(base_color=(0.9, 0.9, 0.9, 1.0), metallic=1.0 if metal else 0.0,
                                     roughness=0.0 if metal else 1.0))
        red = s.add_material(Material(base_color=(1.0, 0.0, 0.0, 1.0), metallic=0.0, roughness=1.0))
        s.add_primitive(quad(0.0, 1.0, material=fm))
        wall = np.array([[-1, 0, -1], [1, 0, -1], [-1, 1, -1], [1, 0, -1], [1, 1, -1], [-1, 1, -1]], np.float32)
        s.add_primitive(Primitive(wall, np.arange(6, dtype=np.uint32), material=red))
        return s

    mirror = oracle.raycast(scene(True), o)[0]
    inert = oracle.raycast(scene(False), o)[0]
    # Floor pixels of the mirror scene carry more red relative to green.
    red_excess = lambda h: float(np.mean(h[..., 0] - h[..., 1]))  # noqa: E731
    assert red_excess(mirror) > red_excess(inert)


def test_transmissive_pane_shows_what_is_behind_it(oracle):
    bg = (0, 0, 0, 255)
    o = RenderOptions(width=32, height=32, shading=ShadingMode.Phong, background=BackgroundColor(bg),
                      light=LightSpec(0.0, 90.0, 1.0), max_ray_depth=3)

    def scene(transmission):
        s = PreparedScene()
        green = s.add_material(Material(base_color=(0.0, 1.0, 0.0, 1.0), metallic=0.0, roughness=1.0))
        pane = s.add_material(Material(base_color=(1.0, 1.0, 1.0, 1.0), metallic=0.0, roughness=0.5,
                                       ext=MaterialExt(transmission=Transmission(transmission))))
        back = np.array([[-2, -2, -1], [2, -2, -1], [-2, 2, -1], [2, -2, -1], [2, 2, -1], [-2, 2, -1]], np.float32)
        s.add_primitive(Primitive(back, np.arange(6, dtype=np.uint32), material=green))
        front = back.copy()
        front[:, 2] = 0.5
        front[:, :2] *= 0.5
        s.add_primitive(Primitive(front, np.arange(6, dtype=np.uint32), material=pane))
        s.add_camera([0.0, 0.0, 3.0], [0.0, 0.0, 0.0], 0.6)
        return s

    see = oracle.raycast(scene(1.0), o.replace(scene_camera=0))[0]
    opaque = oracle.raycast(scene(0.0), o.replace(scene_camera=0))[0]
    c = (slice(12, 20), slice(12, 20))
    assert float(see[c][..., 1].mean() - see[c][..., 0].mean()) > \
        float(opaque[c][..., 1].mean() - opaque[c][..., 0].mean()) + 0.1


def test_unlit_and_emissive_materials(oracle):
    o = RenderOptions(width=16, height=16, shading=ShadingMode.Phong, background=WHITE,
                      light=LightSpec(0.0, 0.0, 0.0))
    s = PreparedScene()
    m = Material(base_color=(0.2, 0.4, 0.6, 1.0), ext=MaterialExt(unlit=True))
    s.add_primitive(Primitive(np.array([[-0.5, -0.5, 0], [0.5, -0.5, 0], [0, 0.5, 0]], np.float32),
                              np.array([0, 1, 2], np.uint32), material=s.add_material(m)))
    hdr = oracle.raycast(s, o)[0]
    center = hdr[8, 8]
    assert np.allclose(center[:3], (0.2, 0.4, 0.6), atol=1e-6)
    e = PreparedScene()
    em = Material(base_color=(0.0, 0.0, 0.0, 1.0), emissive_factor=(0.0, 0.5, 0.0))
    e.add_primitive(Primitive(np.array([[-0.5, -0.5, 0], [0.5, -0.5, 0], [0, 0.5, 0]], np.float32),
                              np.array([0, 1, 2], np.uint32), material=e.add_material(em)))
    assert oracle.raycast(e, o)[0][8, 8, 1] >= 0.5 - 1e-6
