"""Scenes and helpers of the reference's raycast Pbr tests
(tests/raycast_pbr.rs:19-66, 140-210, 267-288, 410-445, 533-575), restated
over this package's PreparedScene, shared by the oracle pins and the device
parity tests."""
import math

import numpy as np

from oxideav_render_b200 import abi, testscenes as ts
from oxideav_render_b200.options import BackgroundColor, RenderOptions, ShadingMode
from oxideav_render_b200.scene import (Camera, Material, MaterialExt, PreparedScene, Primitive, Sampler, Texture,
                                       TextureRef, Transmission, Volume, directional_light)

BG = (0, 0, 0, 255)


def opts(w: int, h: int, **kw) -> RenderOptions:
    """tests/raycast_pbr.rs:19-28: Pbr through the scene's first camera on black."""
    base = dict(width=w, height=h, shading=ShadingMode.Pbr, scene_camera=0, background=BackgroundColor(BG))
    base.update(kw)
    return RenderOptions(**base)


def add(scene: PreparedScene, prim: Primitive, mat: Material, world=None) -> None:
    scene.add_primitive(ts.with_material(prim, scene.add_material(mat)), world)


def unlit(rgb, alpha: float = 1.0, mode: int = abi.PT_ALPHA_OPAQUE) -> Material:
    return Material(base_color=(rgb[0], rgb[1], rgb[2], alpha), alpha_mode=mode, ext=MaterialExt(unlit=True))


def single_quad(mat: Material, world=None) -> PreparedScene:
    s = PreparedScene()
    add(s, ts.quad([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]), mat, world)
    s.add_camera([0.0, 0.0, 2.5], [0.0, 0.0, 0.0], 0.9)
    return s


def floor_quad(half: float, y: float) -> Primitive:
    return ts.quad([[-half, y, half], [half, y, half], [half, y, -half], [-half, y, -half]])


def occluder_scene(occluder: Material, mask_texture: bool = False) -> PreparedScene:
    """A white floor under a single-sided horizontal occluder at y = 1, lit
    straight down (tests/raycast_pbr.rs:267-286)."""
    s = PreparedScene()
    add(s, floor_quad(3.0, 0.0), ts.diffuse_material((0.8, 0.8, 0.8), 1.0))
    if mask_texture:
        px = np.array([[[255, 255, 255, 255], [255, 255, 255, 0]], [[255, 255, 255, 0], [255, 255, 255, 255]]],
                      np.uint8)
        tex = s.add_texture(Texture(px, Sampler(abi.PT_FILTER_NEAREST, abi.PT_MIN_NEAREST)))
        occluder.base_color_texture = TextureRef(tex)
        occluder.alpha_mode = abi.PT_ALPHA_MASK
        occluder.alpha_cutoff = 0.5
    add(s, floor_quad(1.0, 1.0), occluder)
    s.add_light(directional_light((1.0, 1.0, 1.0), 3.0), [0.0, 0.0, 0.0], [0.0, -1.0, 0.0])
    s.add_camera([0.0, 0.5, 4.0], [0.0, 0.0, 0.0], 0.9)
    return s


def metal(roughness: float) -> Material:
    return Material(base_color=(1.0, 1.0, 1.0, 1.0), metallic=1.0, roughness=roughness)


def mirror_scene(floor: Material) -> PreparedScene:
    """A floor of material `floor` in front of an unlit red wall
    (tests/raycast_pbr.rs:410-437)."""
    s = PreparedScene()
    add(s, floor_quad(2.0, 0.0), floor)
    add(s, ts.quad([[-2, 0, -2], [2, 0, -2], [2, 2, -2], [-2, 2, -2]]), unlit((1.0, 0.0, 0.0)))
    s.add_light(directional_light((1.0, 1.0, 1.0), 2.0), [0.0, 0.0, 0.0], [0.3, -1.0, -0.2])
    s.add_camera([0.0, 1.0, 3.0], [0.0, 0.2, -1.0], 0.9)
    return s


def glass(thickness: float, ior: float = 1.5, attenuation_distance=None, attenuation_color=(1.0, 1.0, 1.0)):
    ext = MaterialExt(transmission=Transmission(1.0), ior=ior)
    if thickness > 0.0:
        ext.volume = Volume(thickness=thickness, attenuation_distance=attenuation_distance,
                            attenuation_color=attenuation_color)
    return Material(base_color=(1.0, 1.0, 1.0, 1.0), metallic=0.0, roughness=0.0, ext=ext)


def lens_scene(ball, segments: int = 64, rings: int = 32) -> PreparedScene:
    """An unlit wall at z = -3, red for x < 0 and green for x > 0, a unit
    sphere of material `ball` (None: no sphere) at the origin
    (tests/raycast_pbr.rs:533-553)."""
    s = PreparedScene()
    for x0, x1, c in ((-4.0, 0.0, (1.0, 0.0, 0.0)), (0.0, 4.0, (0.0, 1.0, 0.0))):
        add(s, ts.quad([[x0, -4, -3], [x1, -4, -3], [x1, 4, -3], [x0, 4, -3]]), unlit(c))
    if ball is not None:
        add(s, ts.uv_sphere(1.0, segments, rings), ball)
    s.add_camera([0.0, 0.0, 4.0], [0.0, 0.0, 0.0], 0.7)
    return s


def parallel_mirrors() -> PreparedScene:
    """Two facing perfect mirrors (tests/raycast_pbr.rs:650-668)."""
    s = PreparedScene()
    for z in (-1.0, 1.0):
        a, b = (-2.0, 2.0) if z < 0.0 else (2.0, -2.0)
        add(s, ts.quad([[a, -2, z], [b, -2, z], [b, 2, z], [a, 2, z]]), metal(0.0))
    s.add_camera([0.0, 0.0, 0.5], [0.0, 0.0, -1.0], 0.9)
    return s


def blend_stack(layers: int) -> PreparedScene:
    """`layers` BLEND planes (alpha 0.2, alternating tints) in front of an
    opaque lit wall: deeper than MAX_LAYERS when layers > 64."""
    s = PreparedScene()
    add(s, ts.quad([[-2, -2, -1], [2, -2, -1], [2, 2, -1], [-2, 2, -1]]), ts.diffuse_material((0.7, 0.7, 0.7), 1.0))
    for i in range(layers):
        z = -0.9 + 1.6 * i / max(layers, 1)
        tint = (0.9, 0.3, 0.2) if i % 2 == 0 else (0.2, 0.4, 0.9)
        m = Material(base_color=(tint[0], tint[1], tint[2], 0.2), metallic=0.0, roughness=0.6,
                     alpha_mode=abi.PT_ALPHA_BLEND, double_sided=True)
        add(s, ts.quad([[-1, -1, z], [1, -1, z], [1, 1, z], [-1, 1, z]]), m)
    s.add_light(directional_light((1.0, 1.0, 1.0), 2.0), [0.0, 0.0, 0.0], [-0.3, -0.4, -1.0])
    s.add_camera([0.0, 0.0, 2.5], [0.0, 0.0, 0.0], 0.8)
    return s


def rotate_y(angle: float) -> np.ndarray:
    return ts.rotate_y(angle)


def project(scene: PreparedScene, o: RenderOptions, p) -> tuple:
    """Pixel of world point `p` under the camera `o` selects (perspective)."""
    cam = Camera.resolve(scene, o, o.width, o.height)
    eye, fw = np.asarray(cam.eye, float), np.asarray(cam.forward, float)
    side, up = np.asarray(cam.side, float), np.asarray(cam.up, float)
    v = np.asarray(p, float) - eye
    z = float(v @ fw)
    nx = float(v @ side) / (z * cam.half_w)
    ny = float(v @ up) / (z * cam.half_h)
    return int((nx * 0.5 + 0.5) * o.width), int((1.0 - (ny * 0.5 + 0.5)) * o.height)


def px(img: np.ndarray, xy) -> np.ndarray:
    return img[xy[1], xy[0]]


def luma(p) -> float:
    """testscenes::luma (src/testscenes.rs:1141-1143)."""
    return 0.2126 * float(p[0]) + 0.7152 * float(p[1]) + 0.0722 * float(p[2])


__all__ = ["BG", "opts", "add", "unlit", "single_quad", "floor_quad", "occluder_scene", "metal", "mirror_scene",
           "glass", "lens_scene", "parallel_mirrors", "blend_stack", "rotate_y", "project", "px", "luma", "math"]
