"""Procedural scenes and image metrics.

Geometry builders and reference scenes follow the reference's
src/testscenes.rs (quad :38-56, cuboid :69-81, uv_sphere :109-148,
checker_rgba8 :152-166, cornell_box :305-385, sphere_grid :392-431,
alpha_planes :502-540, shadow_box :547-574, normal_mapped_quad :697-734,
brushed_metal_plate :744-785, iridescent_sphere :793-825,
backlit_leaf :833-867, dispersive_sphere :873-915, material_extensions
:924-1065), the path-tracer test scenes of src/pathtrace.rs (:3348-3705),
and the metrics (mean_abs_error :1069-1080, psnr :1084-1099, region_mean
:1103-1121, region_stddev :1125-1138) plus float-HDR variants.

The benchmark workloads are seeded synthetic scenes:
  * ``cornell_c0``   Cornell-style unit box, 36 triangles, 256x256, 64 spp;
  * ``sphere_grid_c1`` 7x7 UV spheres (64x32 segments, 200,704 triangles)
    over a 512x512 sRGB checker floor, 512x512, 256 spp;
  * ``stress_c2``    1024x1024 fBm heightfield (2,097,152 triangles) plus
    500 UV spheres, 8 emissive triangles, a 512x256 noise environment;
  * ``random_soup``  uniform triangle soups for the batched mix.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from . import abi
from .options import LightSpec, PathTraceOptions, RenderOptions, BackgroundColor
from .scene import (Anisotropy, Camera, Clearcoat, DiffuseTransmission, Iridescence, Material, MaterialExt,
                    PreparedScene, Primitive, Sampler, Specular, Texture, TextureRef, Transmission, Volume,
                    diffuse_material, directional_light, lambert, point_light)

F32 = np.float32


# ----------------------------------------------------------------------------- geometry builders


def _normalize(v):
    v = np.asarray(v, dtype=np.float64)
    n = math.sqrt(float(np.dot(v, v)))
    return v / n if n > 0 else v


def quad(p, uv_scale=(1.0, 1.0)) -> Primitive:
    """Planar quad p0->p1->p2->p3 (CCW from the front), flat normals,
    tangents along p0->p1, UVs p0=(0,1) p1=(1,1) p2=(1,0) p3=(0,0)."""
    p = np.asarray(p, dtype=np.float64)
    e1, e2 = p[1] - p[0], p[3] - p[0]
    n = _normalize(np.cross(e1, e2))
    t = _normalize(e1)
    su, sv = uv_scale
    return Primitive(
        positions=p.astype(F32),
        indices=np.array([0, 1, 2, 0, 2, 3], np.uint32),
        normals=np.tile(n, (4, 1)).astype(F32),
        tangents=np.tile([t[0], t[1], t[2], 1.0], (4, 1)).astype(F32),
        uvs=[np.array([[0.0, sv], [su, sv], [su, 0.0], [0.0, 0.0]], F32)],
    )


def merge(prims: List[Primitive]) -> Primitive:
    pos, nrm, tan, uv, idx = [], [], [], [], []
    base = 0
    for p in prims:
        idx.append(p.indices.astype(np.uint32) + base)
        pos.append(p.positions)
        nrm.append(p.normals)
        tan.append(p.tangents)
        uv.append(p.uvs[0])
        base += p.positions.shape[0]
    return Primitive(np.concatenate(pos), np.concatenate(idx), np.concatenate(nrm), np.concatenate(tan),
                     [np.concatenate(uv)])


def cuboid(mn, mx) -> Primitive:
    """Axis-aligned box with outward faces (24 vertices)."""
    x0, y0, z0 = mn
    x1, y1, z1 = mx
    faces = [
        [[x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]],
        [[x1, y0, z0], [x0, y0, z0], [x0, y1, z0], [x1, y1, z0]],
        [[x1, y0, z1], [x1, y0, z0], [x1, y1, z0], [x1, y1, z1]],
        [[x0, y0, z0], [x0, y0, z1], [x0, y1, z1], [x0, y1, z0]],
        [[x0, y1, z1], [x1, y1, z1], [x1, y1, z0], [x0, y1, z0]],
        [[x0, y0, z0], [x1, y0, z0], [x1, y0, z1], [x0, y0, z1]],
    ]
    return merge([quad(f) for f in faces])


def uv_sphere(radius: float, segments: int, rings: int) -> Primitive:
    """UV sphere: smooth normals, tangents along +u, UVs (u around, v pole to pole)."""
    segments, rings = max(segments, 3), max(rings, 2)
    v = np.arange(rings + 1, dtype=F32) / F32(rings)
    u = np.arange(segments + 1, dtype=F32) / F32(segments)
    theta = (v * F32(math.pi))[:, None]
    phi = (u * F32(2.0 * math.pi))[None, :]
    st, ct = np.sin(theta), np.cos(theta)
    sp, cp = np.sin(phi), np.cos(phi)
    nx = st * cp
    n = np.stack([nx, np.broadcast_to(ct, nx.shape), -st * sp], axis=-1).reshape(-1, 3).astype(F32)
    tg = np.stack([-np.broadcast_to(sp, (rings + 1, segments + 1)), np.zeros((rings + 1, segments + 1), F32),
                   -np.broadcast_to(cp, (rings + 1, segments + 1)), np.ones((rings + 1, segments + 1), F32)],
                  axis=-1).reshape(-1, 4).astype(F32)
    uvs = np.stack(np.broadcast_arrays(u[None, :], v[:, None]), axis=-1).reshape(-1, 2).astype(F32)
    row = segments + 1
    r, s = np.meshgrid(np.arange(rings), np.arange(segments), indexing="ij")
    a = (r * row + s).reshape(-1)
    b = a + row
    idx = np.stack([a, b, a + 1, a + 1, b, b + 1], axis=1).reshape(-1).astype(np.uint32)
    return Primitive((n * F32(radius)).astype(F32), idx, n, tg, [uvs])


def checker_rgba8(size: int, cells: int, a, b) -> np.ndarray:
    cell = max(size // max(cells, 1), 1)
    y, x = np.mgrid[0:size, 0:size]
    even = ((x // cell) + (y // cell)) % 2 == 0
    out = np.where(even[..., None], np.array(a, np.uint8), np.array(b, np.uint8))
    return out.astype(np.uint8)


def translate(t) -> np.ndarray:
    m = np.eye(4)
    m[:3, 3] = t
    return m


def rotate_y(angle: float) -> np.ndarray:
    c, s = math.cos(angle), math.sin(angle)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
    return m


def with_material(prim: Primitive, mat: int) -> Primitive:
    prim.material = mat
    return prim


# ----------------------------------------------------------------------------- reference scenes


def cornell_box() -> PreparedScene:
    """testscenes::cornell_box: [-1,1]^3 room open toward +Z, point light."""
    s = PreparedScene()
    white = s.add_material(diffuse_material((0.75, 0.75, 0.75), 1.0))
    red = s.add_material(diffuse_material((0.65, 0.05, 0.05), 1.0))
    green = s.add_material(diffuse_material((0.12, 0.45, 0.15), 1.0))
    walls = [
        ([[-1, -1, 1], [1, -1, 1], [1, -1, -1], [-1, -1, -1]], white),
        ([[-1, 1, -1], [1, 1, -1], [1, 1, 1], [-1, 1, 1]], white),
        ([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1]], white),
        ([[-1, -1, 1], [-1, -1, -1], [-1, 1, -1], [-1, 1, 1]], red),
        ([[1, -1, -1], [1, -1, 1], [1, 1, 1], [1, 1, -1]], green),
    ]
    for q, m in walls:
        s.add_primitive(with_material(quad(q), m))
    s.add_primitive(with_material(cuboid([-0.6, -1.0, -0.6], [-0.1, 0.2, -0.1]), white))
    s.add_primitive(with_material(cuboid([0.15, -1.0, -0.1], [0.65, -0.4, 0.4]), white))
    s.add_light(point_light((1.0, 0.95, 0.85), 6.0), [0.0, 0.85, 0.0], [0.0, -1.0, 0.0])
    s.add_camera([0.0, 0.0, 3.4], [0.0, 0.0, 0.0], 0.75)
    return s


def sphere_grid(cols: int, rows: int, segments: int = 48, rings: int = 24, base=(0.9, 0.55, 0.25)) -> PreparedScene:
    """testscenes::sphere_grid: metallic 0->1 left to right, roughness 0.05->1 bottom to top."""
    cols, rows = max(cols, 1), max(rows, 1)
    s = PreparedScene()
    sphere = uv_sphere(1.0, segments, rings)
    for r in range(rows):
        for c in range(cols):
            m = Material(base_color=(base[0], base[1], base[2], 1.0),
                         metallic=c / (cols - 1) if cols > 1 else 0.0,
                         roughness=0.05 + 0.95 * r / (rows - 1) if rows > 1 else 0.5)
            mat = s.add_material(m)
            x = (c - (cols - 1) * 0.5) * 2.2
            y = (r - (rows - 1) * 0.5) * 2.2
            s.add_primitive(with_material(Primitive(sphere.positions, sphere.indices, sphere.normals, sphere.tangents,
                                                    sphere.uvs), mat), translate([x, y, 0.0]))
    s.add_light(directional_light((1.0, 1.0, 1.0), 3.0), [0.0, 0.0, 0.0], [0.4, -0.5, -1.0])
    extent = max(cols, rows) * 2.2
    s.add_camera([0.0, 0.0, extent * 1.6], [0.0, 0.0, 0.0], 0.8)
    return s


def shadow_box() -> PreparedScene:
    s = PreparedScene()
    white = s.add_material(diffuse_material((0.8, 0.8, 0.8), 0.9))
    s.add_primitive(with_material(quad([[-3, 0, 3], [3, 0, 3], [3, 0, -3], [-3, 0, -3]]), white))
    s.add_primitive(with_material(cuboid([-0.5, 1.0, -0.5], [0.5, 2.0, 0.5]), white))
    s.add_light(directional_light((1.0, 1.0, 1.0), 3.0), [0.0, 0.0, 0.0], [0.0, -1.0, 0.0])
    s.add_camera([0.0, 6.0, 6.0], [0.0, 0.0, 0.0], 0.9)
    return s


def alpha_planes() -> PreparedScene:
    """Opaque blue back plane, MASK green plane with a cut-out cell, half-width BLEND red plane."""
    s = PreparedScene()

    def unlit(rgb, a, mode):
        return Material(base_color=(rgb[0], rgb[1], rgb[2], a), alpha_mode=mode,
                        ext=MaterialExt(unlit=True))

    blue = s.add_material(unlit((0, 0, 1), 1.0, abi.PT_ALPHA_OPAQUE))
    mask = np.array([[[255, 255, 255, 255], [255, 255, 255, 0]], [[255, 255, 255, 0], [255, 255, 255, 255]]],
                    np.uint8)
    tex = s.add_texture(Texture(mask, Sampler(abi.PT_FILTER_NEAREST, abi.PT_MIN_NEAREST)))
    gm = unlit((0, 1, 0), 1.0, abi.PT_ALPHA_MASK)
    gm.alpha_cutoff = 0.5
    gm.base_color_texture = TextureRef(tex)
    green = s.add_material(gm)
    red = s.add_material(unlit((1, 0, 0), 0.5, abi.PT_ALPHA_BLEND))
    for z, x1, m in [(-1.0, 1.0, blue), (0.0, 1.0, green), (0.5, 0.0, red)]:
        s.add_primitive(with_material(quad([[-1, -1, z], [x1, -1, z], [x1, 1, z], [-1, 1, z]]), m))
    s.add_camera([0.0, 0.0, 1.5], [0.0, 0.0, 0.0], math.pi / 2)
    return s


def normal_mapped_quad(tilt: float) -> PreparedScene:
    s = PreparedScene()
    n = _normalize([tilt, 0.0, 1.0])
    enc = lambda v: int(round((v * 0.5 + 0.5) * 255.0))  # noqa: E731
    tex = s.add_texture(Texture(np.array([[[enc(n[0]), enc(n[1]), enc(n[2]), 255]]], np.uint8)))
    m = diffuse_material((0.8, 0.8, 0.8), 1.0)
    m.normal_texture = TextureRef(tex)
    mat = s.add_material(m)
    s.add_primitive(with_material(quad([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]), mat))
    s.add_light(directional_light((1, 1, 1), 2.0), [0, 0, 0], [-1.0, 0.0, -0.3])
    s.add_camera([0.0, 0.0, 2.5], [0.0, 0.0, 0.0], 0.9)
    return s


def brushed_metal_plate(strength: float, rotation: float) -> PreparedScene:
    s = PreparedScene()
    m = Material(base_color=(0.9, 0.9, 0.9, 1.0), metallic=1.0, roughness=0.35,
                 ext=MaterialExt(anisotropy=Anisotropy(strength, rotation)))
    mat = s.add_material(m)
    s.add_primitive(with_material(quad([[-1, 0, 1], [1, 0, 1], [1, 0, -1], [-1, 0, -1]]), mat))
    s.add_light(point_light((1, 1, 1), 8.0), [0.0, 1.5, 0.0], [0.0, -1.0, 0.0])
    s.add_camera([0.0, 2.0, 0.6], [0.0, 0.0, 0.0], 0.9)
    return s


def iridescent_sphere(iridescence: float, thickness_nm: float) -> PreparedScene:
    s = PreparedScene()
    m = Material(base_color=(0.1, 0.1, 0.1, 1.0), metallic=0.0, roughness=0.25,
                 ext=MaterialExt(iridescence=Iridescence(factor=iridescence, thickness_min=thickness_nm,
                                                         thickness_max=thickness_nm)))
    mat = s.add_material(m)
    s.add_primitive(with_material(uv_sphere(1.0, 48, 24), mat))
    s.add_light(point_light((1, 1, 1), 40.0), [2.0, 3.0, 3.0], [-2.0, -3.0, -3.0])
    s.add_camera([0.0, 0.0, 4.0], [0.0, 0.0, 0.0], 0.7)
    return s


def backlit_leaf(dt: float) -> PreparedScene:
    s = PreparedScene()
    m = Material(base_color=(0.15, 0.5, 0.1, 1.0), metallic=0.0, roughness=1.0, double_sided=True,
                 ext=MaterialExt(diffuse_transmission=DiffuseTransmission(factor=dt, color_factor=(0.6, 0.9, 0.4))))
    mat = s.add_material(m)
    s.add_primitive(with_material(quad([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]), mat))
    s.add_light(point_light((1, 1, 1), 10.0), [0.0, 0.0, -1.5], [0.0, 0.0, 1.0])
    s.add_camera([0.0, 0.0, 3.0], [0.0, 0.0, 0.0], 0.9)
    return s


def _unlit_checker_backdrop(s: PreparedScene, quad_pts, a=(255, 255, 255, 255), b=(0, 0, 0, 255)):
    tex = s.add_texture(Texture(checker_rgba8(64, 8, a, b)))
    bg = s.add_material(Material(base_color_texture=TextureRef(tex), ext=MaterialExt(unlit=True)))
    s.add_primitive(with_material(quad(quad_pts), bg))


def dispersive_sphere(dispersion: float) -> PreparedScene:
    s = PreparedScene()
    _unlit_checker_backdrop(s, [[-4, -4, -2], [4, -4, -2], [4, 4, -2], [-4, 4, -2]])
    g = Material(base_color=(1, 1, 1, 1), metallic=0.0, roughness=0.0,
                 ext=MaterialExt(transmission=Transmission(1.0), volume=Volume(thickness=1.0), ior=1.5,
                                 dispersion=dispersion))
    glass = s.add_material(g)
    s.add_primitive(with_material(uv_sphere(0.8, 48, 24), glass))
    s.add_camera([0.0, 0.0, 3.5], [0.0, 0.0, 0.0], 0.8)
    return s


def material_extensions() -> PreparedScene:
    """Showcase of anisotropy, dispersion, iridescence and diffuse transmission."""
    s = PreparedScene()
    floor = s.add_material(diffuse_material((0.5, 0.5, 0.5), 1.0))
    s.add_primitive(with_material(quad([[-4, -1, 4], [4, -1, 4], [4, -1, -4], [-4, -1, -4]]), floor))
    _unlit_checker_backdrop(s, [[-4, -1, -3], [4, -1, -3], [4, 5, -3], [-4, 5, -3]], (230, 230, 230, 255),
                            (20, 20, 20, 255))
    plate = s.add_material(Material(base_color=(0.9, 0.9, 0.9, 1.0), metallic=1.0, roughness=0.35,
                                    ext=MaterialExt(anisotropy=Anisotropy(0.9, 0.0))))
    s.add_primitive(with_material(quad([[-2.4, -0.95, 0.9], [-0.8, -0.95, 0.9], [-0.8, -0.95, -0.7],
                                        [-2.4, -0.95, -0.7]]), plate))
    glass = s.add_material(Material(base_color=(1, 1, 1, 1), metallic=0.0, roughness=0.0,
                                    ext=MaterialExt(transmission=Transmission(1.0), volume=Volume(thickness=1.0),
                                                    ior=1.5, dispersion=1.0)))
    s.add_primitive(with_material(uv_sphere(0.45, 48, 24), glass), translate([-1.6, -0.2, 0.6]))
    irid = s.add_material(Material(base_color=(0.8, 0.8, 0.8, 1.0), metallic=0.0, roughness=0.15,
                                   ext=MaterialExt(iridescence=Iridescence(factor=1.0, thickness_min=550.0,
                                                                           thickness_max=550.0))))
    s.add_primitive(with_material(uv_sphere(0.6, 48, 24), irid), translate([0.0, -0.4, 0.0]))
    leaf = s.add_material(Material(base_color=(0.15, 0.5, 0.1, 1.0), metallic=0.0, roughness=1.0, double_sided=True,
                                   ext=MaterialExt(diffuse_transmission=DiffuseTransmission(
                                       factor=0.8, color_factor=(0.6, 0.9, 0.4)))))
    s.add_primitive(with_material(quad([[0.9, -0.9, 0.3], [2.1, -0.9, 0.3], [2.1, 0.5, 0.3], [0.9, 0.5, 0.3]]), leaf))
    s.add_light(point_light((1.0, 0.95, 0.8), 6.0), [1.5, -0.2, -0.8], [0.0, 0.0, 1.0])
    s.add_light(point_light((1, 1, 1), 40.0), [0.0, 2.5, 2.0], [0.0, -1.0, -0.5])
    s.add_camera([0.0, 0.6, 4.5], [0.0, -0.3, 0.0], 0.8)
    return s


# -- path-tracer test scenes (src/pathtrace.rs:3348-3705) ----------------------


def furnace_scene(rho: float, le: float) -> PreparedScene:
    """Closed box of double-sided emissive Lambert walls: L = Le / (1 - rho)."""
    s = PreparedScene()
    m = lambert((rho, rho, rho))
    m.emissive_factor = (le, le, le)
    m.double_sided = True
    mat = s.add_material(m)
    s.add_primitive(with_material(cuboid([-1, -1, -1], [1, 1, 1]), mat))
    s.add_camera([0.2, 0.1, 0.4], [0.0, -0.3, -1.0], 1.2)
    return s


def area_light_scene(roughness: float, metallic: float) -> PreparedScene:
    s = PreparedScene()
    fm = diffuse_material((0.8, 0.8, 0.8), roughness)
    fm.metallic = metallic
    floor = s.add_material(fm)
    lm = lambert((0, 0, 0))
    lm.emissive_factor = (4.0, 4.0, 4.0)
    light = s.add_material(lm)
    s.add_primitive(with_material(quad([[-2, 0, 2], [2, 0, 2], [2, 0, -2], [-2, 0, -2]]), floor))
    s.add_primitive(with_material(quad([[-0.5, 1, -0.5], [0.5, 1, -0.5], [0.5, 1, 0.5], [-0.5, 1, 0.5]]), light))
    s.add_camera([0.0, 2.5, 3.0], [0.0, 0.0, 0.0], 0.9)
    return s


def glass_scene(volume: bool) -> PreparedScene:
    s = PreparedScene()
    g = diffuse_material((1, 1, 1), 0.0)
    g.ext.transmission = Transmission(1.0)
    if volume:
        g.ext.volume = Volume(thickness=1.0, attenuation_distance=1.0, attenuation_color=(0.5, 0.5, 0.5))
    gm = s.add_material(g)
    lm = lambert((0, 0, 0))
    lm.emissive_factor = (1.0, 1.0, 1.0)
    em = s.add_material(lm)
    s.add_primitive(with_material(cuboid([-0.5] * 3, [0.5] * 3), gm))
    s.add_primitive(with_material(quad([[-3, -3, -2], [3, -3, -2], [3, 3, -2], [-3, 3, -2]]), em))
    s.add_camera([0.0, 0.0, 4.0], [0.0, 0.0, 0.0], 0.15)
    return s


def lambert_plane(rho: float = 0.5, cam=((0.0, 2.0, 0.01), 0.4)) -> PreparedScene:
    s = PreparedScene()
    mat = s.add_material(lambert((rho, rho, rho)))
    s.add_primitive(with_material(quad([[-1, 0, 1], [1, 0, 1], [1, 0, -1], [-1, 0, -1]]), mat))
    s.add_camera(cam[0], [0.0, 0.0, 0.0], cam[1])
    return s


def point_light_plane() -> PreparedScene:
    s = lambert_plane(1.0, ((0.0, 3.0, 0.001), 0.05))
    s.add_light(point_light((1, 1, 1), 4.0), [0.0, 1.0, 0.0], [0.0, -1.0, 0.0])
    return s


def pt_opts(w: int, spp: int, bounces: int, h: Optional[int] = None, **kw) -> RenderOptions:
    """The path-tracer tests' option helper (src/pathtrace.rs:2819-2838)."""
    pt = PathTraceOptions(samples_per_pixel=spp, max_bounces=bounces, **{k: v for k, v in kw.items()
                                                                         if k in ("rr_start", "clamp", "seed",
                                                                                  "strategy")})
    rest = {k: v for k, v in kw.items() if k not in ("rr_start", "clamp", "seed", "strategy")}
    base = dict(width=w, height=h if h is not None else w, scene_camera=0, ambient=0.0,
                light=LightSpec(intensity=0.0), background=BackgroundColor((0, 0, 0, 255)), path_trace=pt)
    base.update(rest)
    return RenderOptions(**base)


# ----------------------------------------------------------------------------- benchmark workloads


def cornell_c0() -> Tuple[PreparedScene, RenderOptions]:
    """Cornell-style unit box: 5 diffuse quads (white 0.73, red, green), a
    0.25 x 0.25 ceiling emitter (17, 12, 4), two boxes rotated +-18 deg
    (36 triangles); 40 deg pinhole; 256x256, 64 spp, 8 bounces, clamp 0,
    black sky, seed 0, no fallback light."""
    s = PreparedScene()
    white = s.add_material(diffuse_material((0.73, 0.73, 0.73), 1.0))
    red = s.add_material(diffuse_material((0.65, 0.05, 0.05), 1.0))
    green = s.add_material(diffuse_material((0.12, 0.45, 0.15), 1.0))
    lm = lambert((0.0, 0.0, 0.0))
    lm.emissive_factor = (17.0, 12.0, 4.0)
    light = s.add_material(lm)
    h = 0.5
    walls = [
        ([[-h, -h, h], [h, -h, h], [h, -h, -h], [-h, -h, -h]], white),   # floor (+Y)
        ([[-h, h, -h], [h, h, -h], [h, h, h], [-h, h, h]], white),       # ceiling (-Y)
        ([[-h, -h, -h], [h, -h, -h], [h, h, -h], [-h, h, -h]], white),   # back (+Z)
        ([[-h, -h, h], [-h, -h, -h], [-h, h, -h], [-h, h, h]], red),     # left (+X)
        ([[h, -h, -h], [h, -h, h], [h, h, h], [h, h, -h]], green),       # right (-X)
    ]
    for q, m in walls:
        s.add_primitive(with_material(quad(q), m))
    e, y = 0.125, h - 1.0e-3
    s.add_primitive(with_material(quad([[-e, y, -e], [e, y, -e], [e, y, e], [-e, y, e]]), light))
    tall = cuboid([-0.15, -h, -0.15], [0.15, 0.1, 0.15])
    short = cuboid([-0.15, -h, -0.15], [0.15, -0.2, 0.15])
    s.add_primitive(with_material(tall, white), translate([-0.17, 0, -0.15]) @ rotate_y(math.radians(18.0)))
    s.add_primitive(with_material(short, white), translate([0.17, 0, 0.12]) @ rotate_y(math.radians(-18.0)))
    s.add_camera([0.0, 0.0, 1.9], [0.0, 0.0, 0.0], math.radians(40.0))
    opts = RenderOptions(width=256, height=256, scene_camera=0, ambient=0.0, light=LightSpec(intensity=0.0),
                         background=BackgroundColor((0, 0, 0, 255)),
                         path_trace=PathTraceOptions(samples_per_pixel=64, max_bounces=8, clamp=0.0, seed=0))
    return s, opts


def sphere_grid_c1(width: int = 512, spp: int = 256) -> Tuple[PreparedScene, RenderOptions]:
    """7x7 UV spheres (64x32 segments, 4,096 triangles each) with metallic
    0->1 across rows and roughness 0.05->1 across columns, base (0.8, 0.2,
    0.2); a checker floor with a 512^2 sRGB RGBA8 texture (trilinear mips);
    one directional (intensity 3) and one point light (intensity 50); sky
    0.3; 512x512, 256 spp, 8 bounces."""
    s = PreparedScene()
    sphere = uv_sphere(1.0, 64, 32)
    n = 7
    for r in range(n):
        for c in range(n):
            m = Material(base_color=(0.8, 0.2, 0.2, 1.0), metallic=r / (n - 1), roughness=0.05 + 0.95 * c / (n - 1))
            mat = s.add_material(m)
            s.add_primitive(with_material(Primitive(sphere.positions, sphere.indices, sphere.normals,
                                                    sphere.tangents, sphere.uvs), mat),
                            translate([(c - 3) * 2.2, (r - 3) * 2.2, 0.0]))
    tex = s.add_texture(Texture(checker_rgba8(512, 16, (230, 230, 230, 255), (40, 40, 40, 255))))
    fl = diffuse_material((1.0, 1.0, 1.0), 0.8)
    fl.base_color_texture = TextureRef(tex)
    floor = s.add_material(fl)
    y = -3 * 2.2 - 1.05
    s.add_primitive(with_material(quad([[-12, y, 12], [12, y, 12], [12, y, -12], [-12, y, -12]], (6.0, 6.0)), floor))
    s.add_light(directional_light((1, 1, 1), 3.0), [0, 0, 0], [0.4, -0.5, -1.0])
    s.add_light(point_light((1.0, 0.9, 0.8), 50.0), [0.0, 9.0, 6.0], [0.0, -1.0, 0.0])
    s.add_camera([0.0, 2.0, 7 * 2.2 * 1.6], [0.0, -1.0, 0.0], 0.8)
    opts = RenderOptions(width=width, height=width, scene_camera=0, ambient=0.3,
                         background=BackgroundColor((0, 0, 0, 255)),
                         path_trace=PathTraceOptions(samples_per_pixel=spp, max_bounces=8))
    return s, opts


def _fbm(n: int, octaves: int, rng: np.random.Generator) -> np.ndarray:
    """fBm value noise on an (n+1)^2 lattice in [0, 1)."""
    out = np.zeros((n + 1, n + 1), np.float64)
    amp, freq, norm = 1.0, 4, 0.0
    g = np.linspace(0.0, 1.0, n + 1)
    for _ in range(octaves):
        lat = rng.random((freq + 1, freq + 1))
        x = g * freq
        i0 = np.minimum(np.floor(x).astype(int), freq - 1)
        f = x - i0
        f = f * f * (3 - 2 * f)
        a = lat[i0][:, i0]
        b = lat[i0][:, i0 + 1]
        c = lat[i0 + 1][:, i0]
        d = lat[i0 + 1][:, i0 + 1]
        fy, fx = f[:, None], f[None, :]
        out += amp * ((a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy)
        norm += amp
        amp *= 0.5
        freq *= 2
    return out / norm


def heightfield_primitive(n: int, amplitude: float, rng) -> Primitive:
    h = (_fbm(n, 5, rng) * amplitude).astype(np.float64)
    g = np.linspace(0.0, 1.0, n + 1)
    xs, zs = np.meshgrid(g, g)
    pos = np.stack([xs, h, zs], axis=-1).reshape(-1, 3).astype(F32)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    a = (i * (n + 1) + j).reshape(-1)
    b = a + 1
    c = a + (n + 1)
    d = c + 1
    idx = np.stack([a, c, b, b, c, d], axis=1).reshape(-1).astype(np.uint32)
    return Primitive(pos, idx)


def env_noise(width: int, height: int, rng) -> np.ndarray:
    """Smooth-noise equirect environment (f32 RGBA), brighter toward +Y."""
    lat = rng.random((9, 17, 3))
    v = np.linspace(0, 8, height)[:, None]
    u = np.linspace(0, 16, width)[None, :]
    i0 = np.minimum(np.floor(v).astype(int), 7)
    j0 = np.minimum(np.floor(u).astype(int), 15)
    fv, fu = v - i0, u - j0
    c = (lat[i0, j0] * ((1 - fu) * (1 - fv))[..., None] + lat[i0, j0 + 1] * (fu * (1 - fv))[..., None]
         + lat[i0 + 1, j0] * ((1 - fu) * fv)[..., None] + lat[i0 + 1, j0 + 1] * (fu * fv)[..., None])
    sky = 0.3 + 1.2 * np.clip(1.0 - np.linspace(0, 1, height), 0, 1)[:, None, None]
    rgb = (c * 0.6 + 0.2) * sky
    return np.concatenate([rgb, np.ones((height, width, 1))], axis=-1).astype(F32)


def stress_c2(width: int = 1920, height: int = 1080, spp: int = 64, grid: int = 1024, spheres: int = 500,
              seed: int = 2026):
    """BVH stress scene: a grid x grid fBm heightfield (5 octaves, amplitude
    0.1) plus `spheres` UV spheres (64x32, radius U(0.01, 0.05)) with
    materials uniform over {diffuse, GGX metal roughness U(0,1), dielectric
    transmission 1 ior 1.5, clearcoat}; 8 emissive triangles with emission
    U(5, 20); a 512x256 smooth-noise environment. Returns (scene, options,
    environment pixels)."""
    rng = np.random.default_rng(seed)
    s = PreparedScene()
    ground = s.add_material(diffuse_material((0.55, 0.5, 0.45), 0.9))
    s.add_primitive(with_material(heightfield_primitive(grid, 0.1, rng), ground))
    sphere = uv_sphere(1.0, 64, 32)
    for _ in range(spheres):
        kind = int(rng.integers(0, 4))
        col = tuple(float(v) for v in rng.uniform(0.2, 0.9, 3))
        if kind == 0:
            m = diffuse_material(col, 1.0)
        elif kind == 1:
            m = Material(base_color=col + (1.0,), metallic=1.0, roughness=float(rng.uniform(0, 1)))
        elif kind == 2:
            m = Material(base_color=(1, 1, 1, 1), metallic=0.0, roughness=0.05,
                         ext=MaterialExt(transmission=Transmission(1.0), ior=1.5))
        else:
            m = Material(base_color=col + (1.0,), metallic=0.0, roughness=0.6,
                         ext=MaterialExt(clearcoat=Clearcoat(factor=1.0, roughness=0.1)))
        mat = s.add_material(m)
        r = float(rng.uniform(0.01, 0.05))
        p = rng.uniform([0.05, 0.1, 0.05], [0.95, 0.35, 0.95])
        w = np.diag([r, r, r, 1.0])
        w[:3, 3] = p
        s.add_primitive(with_material(Primitive(sphere.positions, sphere.indices, sphere.normals, sphere.tangents,
                                                sphere.uvs), mat), w)
    for _ in range(8):
        le = float(rng.uniform(5, 20))
        lm = lambert((0, 0, 0))
        lm.emissive_factor = (le, le * 0.9, le * 0.8)
        lm.double_sided = True
        mat = s.add_material(lm)
        c = rng.uniform([0.1, 0.4, 0.1], [0.9, 0.6, 0.9])
        tri = (c + rng.uniform(-0.04, 0.04, (3, 3))).astype(F32)
        s.add_primitive(Primitive(tri, np.array([0, 1, 2], np.uint32), material=mat))
    s.add_camera([0.5, 0.55, 1.45], [0.5, 0.05, 0.45], 0.75)
    opts = RenderOptions(width=width, height=height, scene_camera=0, ambient=0.0, light=LightSpec(intensity=0.0),
                         background=BackgroundColor((0, 0, 0, 255)),
                         path_trace=PathTraceOptions(samples_per_pixel=spp, max_bounces=8))
    return s, opts, env_noise(512, 256, rng)


def random_soup(tris: int, seed: int) -> PreparedScene:
    """`tris` uniform triangles of edge U(0.005, 0.05) in the unit cube with
    random diffuse / metal / dielectric materials, lit by one emitter quad and
    a point light."""
    rng = np.random.default_rng(seed)
    s = PreparedScene()
    mats = [s.add_material(diffuse_material((0.7, 0.6, 0.5), 1.0)),
            s.add_material(Material(base_color=(0.9, 0.8, 0.6, 1.0), metallic=1.0, roughness=0.3)),
            s.add_material(Material(base_color=(1, 1, 1, 1), metallic=0.0, roughness=0.1,
                                    ext=MaterialExt(transmission=Transmission(1.0))))]
    c = rng.random((tris, 1, 3))
    edge = rng.uniform(0.005, 0.05, (tris, 1, 1))
    d = rng.normal(size=(tris, 3, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    pos = (c + d * edge).astype(F32)
    which = rng.integers(0, 3, tris)
    for k, m in enumerate(mats):
        sel = pos[which == k].reshape(-1, 3)
        if sel.shape[0]:
            s.add_primitive(Primitive(np.ascontiguousarray(sel), material=m))
    lm = lambert((0, 0, 0))
    lm.emissive_factor = (8.0, 8.0, 8.0)
    lmat = s.add_material(lm)
    s.add_primitive(with_material(quad([[0.3, 1.2, 0.3], [0.7, 1.2, 0.3], [0.7, 1.2, 0.7], [0.3, 1.2, 0.7]]), lmat))
    s.add_light(point_light((1, 1, 1), 2.0), [0.5, 1.5, 1.5], [0, -1, -1])
    s.add_camera([0.5, 0.5, 2.2], [0.5, 0.5, 0.5], 0.8)
    return s


# ----------------------------------------------------------------------------- metrics


def mean_abs_error(a: np.ndarray, b: np.ndarray) -> float:
    """RGB mean absolute error on RGBA8 images (0..255 scale)."""
    assert a.shape == b.shape, "size mismatch"
    return float(np.mean(np.abs(a[..., :3].astype(np.int64) - b[..., :3].astype(np.int64))))


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    """PSNR over RGB of RGBA8 images (inf for identical images)."""
    assert a.shape == b.shape, "size mismatch"
    d = a[..., :3].astype(np.float64) - b[..., :3].astype(np.float64)
    se = float(np.mean(d * d))
    return math.inf if se == 0.0 else 10.0 * math.log10(255.0 * 255.0 / se)


def region_mean(img: np.ndarray, x0: int, y0: int, x1: int, y1: int) -> np.ndarray:
    r = img[y0:min(y1, img.shape[0]), x0:min(x1, img.shape[1])].astype(np.float64)
    return r.reshape(-1, img.shape[-1]).mean(axis=0) if r.size else np.zeros(img.shape[-1])


def region_stddev(img: np.ndarray, x0: int, y0: int, x1: int, y1: int) -> float:
    r = img[y0:min(y1, img.shape[0]), x0:min(x1, img.shape[1])].astype(np.float64)
    if r.size == 0:
        return 0.0
    l = 0.2126 * r[..., 0] + 0.7152 * r[..., 1] + 0.0722 * r[..., 2]
    return float(l.std())


def hdr_mae(a: np.ndarray, b: np.ndarray) -> float:
    """Per-channel mean absolute error of two float HDR RGBA images (RGB)."""
    return float(np.mean(np.abs(a[..., :3].astype(np.float64) - b[..., :3].astype(np.float64))))


def hdr_psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    """PSNR of two float HDR images over RGB with the given peak (1.0 = display white)."""
    d = a[..., :3].astype(np.float64) - b[..., :3].astype(np.float64)
    se = float(np.mean(d * d))
    return math.inf if se == 0.0 else 10.0 * math.log10(peak * peak / se)
