"""Host-side scene input: the flattened `PreparedScene` the library consumes.

The reference turns a glTF-like `Scene3D` into a `PreparedScene`
(src/prepare.rs:1098-1234): world-space, de-indexed triangle `DrawItem`s with
CCW front faces, a resolved material table (`PreparedMaterial::from_material`,
:625-670, plus the fallback material :602-623), a texture table, world-space
punctual lights (or the options' fallback light, :1197-1204, built by
`PreparedLight::from_light_spec` :848-863) and scene-camera instances.
This module builds exactly that data with numpy and packs it into the
`pt_scene_desc` ABI struct (include/pt_b200.h). Primitives are
instanced with the same rules as `flatten_primitive` (:1352-1517): normal
matrix for normals, winding flip for mirroring transforms, flat face normals
when a primitive has none.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .options import LightSpec, Projection, RenderOptions

# ----------------------------------------------------------------------------- textures


@dataclass
class Sampler:
    """glTF sampler with mesh3d's effective filters already applied
    (defaults: bilinear magnification, trilinear minification, REPEAT)."""

    mag_filter: int = abi.PT_FILTER_LINEAR
    min_filter: int = abi.PT_MIN_LINEAR_MIP_LINEAR
    wrap_s: int = abi.PT_WRAP_REPEAT
    wrap_t: int = abi.PT_WRAP_REPEAT


@dataclass
class Texture:
    """A decoded image: (h, w, 4) uint8 RGBA8 or float32 RGBA."""

    pixels: np.ndarray
    sampler: Sampler = field(default_factory=Sampler)


@dataclass
class TextureTransform:
    """KHR_texture_transform: uv' = T(offset) * R(rotation) * S(scale) * uv."""

    offset: tuple = (0.0, 0.0)
    rotation: float = 0.0
    scale: tuple = (1.0, 1.0)
    tex_coord: Optional[int] = None

    def is_identity(self) -> bool:
        return self.offset == (0.0, 0.0) and self.rotation == 0.0 and self.scale == (1.0, 1.0)

    def matrix(self) -> list:
        c, s = math.cos(self.rotation), math.sin(self.rotation)
        sx, sy = self.scale
        return [c * sx, s * sy, self.offset[0], -s * sx, c * sy, self.offset[1]]


@dataclass
class TextureRef:
    texture: int
    tex_coord: int = 0
    transform: Optional[TextureTransform] = None

    def effective_uv_set(self) -> int:
        if self.transform is not None and self.transform.tex_coord is not None:
            return self.transform.tex_coord
        return self.tex_coord


# ----------------------------------------------------------------------------- materials


@dataclass
class Specular:
    factor: float = 1.0
    factor_texture: Optional[TextureRef] = None
    color_factor: tuple = (1.0, 1.0, 1.0)
    color_texture: Optional[TextureRef] = None


@dataclass
class Transmission:
    factor: float = 0.0
    factor_texture: Optional[TextureRef] = None


@dataclass
class Volume:
    thickness: float = 0.0
    thickness_texture: Optional[TextureRef] = None
    attenuation_distance: Optional[float] = None
    attenuation_color: tuple = (1.0, 1.0, 1.0)

    def effective_attenuation_distance(self) -> float:
        d = self.attenuation_distance
        return math.inf if d is None else d


@dataclass
class Clearcoat:
    factor: float = 0.0
    factor_texture: Optional[TextureRef] = None
    roughness: float = 0.0
    roughness_texture: Optional[TextureRef] = None
    normal_texture: Optional[TextureRef] = None
    normal_scale: float = 1.0


@dataclass
class Sheen:
    color_factor: tuple = (0.0, 0.0, 0.0)
    color_texture: Optional[TextureRef] = None
    roughness: float = 0.0
    roughness_texture: Optional[TextureRef] = None


@dataclass
class Anisotropy:
    strength: float = 0.0
    rotation: float = 0.0
    texture: Optional[TextureRef] = None


@dataclass
class Iridescence:
    factor: float = 0.0
    factor_texture: Optional[TextureRef] = None
    ior: float = 1.3
    thickness_min: float = 100.0
    thickness_max: float = 400.0
    thickness_texture: Optional[TextureRef] = None


@dataclass
class DiffuseTransmission:
    factor: float = 0.0
    factor_texture: Optional[TextureRef] = None
    color_factor: tuple = (1.0, 1.0, 1.0)
    color_texture: Optional[TextureRef] = None


@dataclass
class MaterialExt:
    unlit: bool = False
    emissive_strength: Optional[float] = None
    ior: Optional[float] = None
    specular: Optional[Specular] = None
    transmission: Optional[Transmission] = None
    volume: Optional[Volume] = None
    clearcoat: Optional[Clearcoat] = None
    sheen: Optional[Sheen] = None
    anisotropy: Optional[Anisotropy] = None
    iridescence: Optional[Iridescence] = None
    diffuse_transmission: Optional[DiffuseTransmission] = None
    dispersion: Optional[float] = None


ALPHA_OPAQUE, ALPHA_MASK, ALPHA_BLEND = abi.PT_ALPHA_OPAQUE, abi.PT_ALPHA_MASK, abi.PT_ALPHA_BLEND


@dataclass
class Material:
    """glTF metallic-roughness material (glTF defaults)."""

    base_color: tuple = (1.0, 1.0, 1.0, 1.0)
    base_color_texture: Optional[TextureRef] = None
    metallic: float = 1.0
    roughness: float = 1.0
    metallic_roughness_texture: Optional[TextureRef] = None
    normal_texture: Optional[TextureRef] = None
    normal_scale: float = 1.0
    occlusion_texture: Optional[TextureRef] = None
    occlusion_strength: float = 1.0
    emissive_factor: tuple = (0.0, 0.0, 0.0)
    emissive_texture: Optional[TextureRef] = None
    alpha_mode: int = ALPHA_OPAQUE
    alpha_cutoff: float = 0.5
    double_sided: bool = False
    ext: MaterialExt = field(default_factory=MaterialExt)


def diffuse_material(rgb, roughness: float) -> Material:
    """testscenes::diffuse_material (src/testscenes.rs:170-177)."""
    return Material(base_color=(rgb[0], rgb[1], rgb[2], 1.0), metallic=0.0, roughness=roughness)


def lambert(rgb) -> Material:
    """Dielectric with KHR_materials_specular factor 0 (pathtrace tests :2810-2817)."""
    m = diffuse_material(rgb, 1.0)
    m.ext.specular = Specular(factor=0.0)
    return m


def _fin(v: float, d: float) -> float:
    return v if math.isfinite(v) else d


def _clamp(v: float, lo: float, hi: float) -> float:
    return min(max(v, lo), hi)


# ----------------------------------------------------------------------------- geometry


@dataclass
class Primitive:
    """Indexed triangle primitive in local space."""

    positions: np.ndarray                  # (n, 3) float32
    indices: Optional[np.ndarray] = None   # (m,) uint32, triangles
    normals: Optional[np.ndarray] = None   # (n, 3)
    tangents: Optional[np.ndarray] = None  # (n, 4)
    uvs: List[np.ndarray] = field(default_factory=list)  # each (n, 2)
    colors: Optional[np.ndarray] = None    # (n, 4)
    material: Optional[int] = None


@dataclass
class DrawItem:
    """De-indexed world-space triangle item (src/prepare.rs:170-211)."""

    positions: np.ndarray       # (3t, 3) float32
    normals: Optional[np.ndarray]
    has_vertex_normals: bool
    tangents: Optional[np.ndarray]
    uvs: List[Optional[np.ndarray]]
    colors: Optional[np.ndarray]
    material: int

    @property
    def triangle_count(self) -> int:
        return self.positions.shape[0] // 3


@dataclass
class Light:
    kind: int
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    range: Optional[float] = None
    inner_cone_angle: float = 0.0
    outer_cone_angle: float = math.pi / 4


def point_light(color=(1.0, 1.0, 1.0), intensity=1.0, range=None) -> Light:
    return Light(abi.PT_LIGHT_POINT, tuple(color), intensity, range)


def directional_light(color=(1.0, 1.0, 1.0), intensity=1.0) -> Light:
    return Light(abi.PT_LIGHT_DIRECTIONAL, tuple(color), intensity)


def spot_light(color=(1.0, 1.0, 1.0), intensity=1.0, range=None, inner=0.0, outer=math.pi / 4) -> Light:
    return Light(abi.PT_LIGHT_SPOT, tuple(color), intensity, range, inner, outer)


@dataclass
class PlacedLight:
    """PreparedLight (src/prepare.rs:687-713)."""

    kind: int
    color: tuple
    intensity: float
    position: tuple
    direction: tuple
    range: Optional[float]
    inner_cone_angle: float
    outer_cone_angle: float


@dataclass
class SceneCamera:
    """A glTF camera placed by a node world matrix (4x4, column vectors)."""

    world: np.ndarray
    perspective: bool = True
    yfov: float = math.pi / 3
    ymag: float = 1.0
    znear: float = 0.01
    zfar: Optional[float] = None  # None: infinite (perspective) / unset


def _normalise(v):
    v = np.asarray(v, dtype=np.float64)
    n = float(np.sqrt(np.dot(v, v)))
    return v / n if n >= 1.1920929e-07 else np.zeros(3)


def look_at_world(eye, target) -> np.ndarray:
    """Node world matrix placing a camera / light at `eye` whose local -Z
    points at `target` (testscenes::look_rotation, src/testscenes.rs:215-270)."""
    f = _normalise(np.subtract(target, eye))
    up = np.array([0.0, 0.0, -1.0]) if abs(f[1]) > 0.99 else np.array([0.0, 1.0, 0.0])
    z = -f
    x = _normalise(np.cross(up, z))
    y = np.cross(z, x)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = x, y, z, eye
    return m


class PreparedScene:
    """The flattened scene (src/prepare.rs:1028-1048)."""

    def __init__(self):
        self.items: List[DrawItem] = []
        self.materials: List[Material] = []
        self.textures: List[Optional[Texture]] = []
        self.scene_lights: List[PlacedLight] = []
        self.cameras: List[SceneCamera] = []
        self._bounds = None

    # -- building -------------------------------------------------------------
    def add_material(self, m: Material) -> int:
        self.materials.append(m)
        return len(self.materials) - 1

    def add_texture(self, t: Optional[Texture]) -> int:
        self.textures.append(t)
        return len(self.textures) - 1

    def add_light(self, light: Light, position, direction) -> None:
        d = _normalise(direction)
        if float(np.dot(d, d)) < 0.5:
            d = np.array([0.0, 0.0, -1.0])
        fin = lambda v: max(v, 0.0) if math.isfinite(v) else 0.0  # noqa: E731
        rng = light.range if (light.range is not None and math.isfinite(light.range) and light.range > 0) else None
        outer, inner = light.outer_cone_angle, light.inner_cone_angle
        if light.kind == abi.PT_LIGHT_SPOT:
            outer = _clamp(outer, 1.0e-4, math.pi / 2) if math.isfinite(outer) else math.pi / 4
            inner = _clamp(inner, 0.0, outer) if math.isfinite(inner) else 0.0
        else:
            outer, inner = 0.0, 0.0
            if light.kind == abi.PT_LIGHT_DIRECTIONAL:
                rng = None
        self.scene_lights.append(PlacedLight(
            light.kind, tuple(fin(c) for c in light.color), fin(light.intensity),
            tuple(float(v) for v in position), tuple(float(v) for v in d), rng, inner, outer))

    def add_camera(self, eye, target, yfov: float) -> int:
        self.cameras.append(SceneCamera(look_at_world(np.asarray(eye, float), np.asarray(target, float)), True, yfov))
        return len(self.cameras) - 1

    def add_primitive(self, prim: Primitive, world: Optional[np.ndarray] = None) -> None:
        """Instance `prim` at `world` (flatten_primitive, src/prepare.rs:1352-1517)."""
        world = np.eye(4) if world is None else np.asarray(world, np.float64)
        nv = prim.positions.shape[0]
        if nv == 0:
            return
        m3 = world[:3, :3]
        pos = (prim.positions.astype(np.float64) @ m3.T + world[:3, 3]).astype(np.float32)
        det = float(np.linalg.det(m3))
        idx = prim.indices if prim.indices is not None else np.arange(nv, dtype=np.uint32)
        tri = np.asarray(idx, dtype=np.int64).reshape(-1, 3)
        ok = np.all((tri >= 0) & (tri < nv), axis=1)
        tri = tri[ok]
        finite = np.all(np.isfinite(pos), axis=1)
        tri = tri[np.all(finite[tri], axis=1)]
        if det < 0:
            tri = tri[:, [0, 2, 1]]
        if tri.shape[0] == 0:
            return
        corners = tri.reshape(-1)
        positions = np.ascontiguousarray(pos[corners])
        if prim.normals is not None and prim.normals.shape[0] == nv:
            nm = np.linalg.inv(m3).T if abs(det) > 1e-20 else np.eye(3)
            n = prim.normals.astype(np.float64) @ nm.T
            ln = np.linalg.norm(n, axis=1, keepdims=True)
            n = np.where(ln >= 1.1920929e-07, n / np.maximum(ln, 1e-30), 0.0)
            normals = np.ascontiguousarray(n.astype(np.float32)[corners])
            has_vn = True
        else:
            p = positions.reshape(-1, 3, 3).astype(np.float64)
            fn = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
            ln = np.linalg.norm(fn, axis=1, keepdims=True)
            fn = np.where(ln >= 1.1920929e-07, fn / np.maximum(ln, 1e-30), 0.0)
            normals = np.ascontiguousarray(np.repeat(fn, 3, axis=0).astype(np.float32))
            has_vn = False
        tangents = None
        if prim.tangents is not None and prim.tangents.shape[0] == nv:
            t = prim.tangents[:, :3].astype(np.float64) @ m3.T
            lt = np.linalg.norm(t, axis=1, keepdims=True)
            t = np.where(lt >= 1.1920929e-07, t / np.maximum(lt, 1e-30), 0.0)
            w = np.where(prim.tangents[:, 3] < 0, -1.0, 1.0) * (-1.0 if det < 0 else 1.0)
            tangents = np.ascontiguousarray(np.concatenate([t, w[:, None]], axis=1).astype(np.float32)[corners])
        uvs: List[Optional[np.ndarray]] = []
        for s in range(abi.PT_MAX_UV_SETS):
            if s < len(prim.uvs) and prim.uvs[s] is not None and prim.uvs[s].shape[0] == nv:
                uvs.append(np.ascontiguousarray(prim.uvs[s].astype(np.float32)[corners]))
            else:
                uvs.append(None)
        colors = None
        if prim.colors is not None and prim.colors.shape[0] == nv:
            colors = np.ascontiguousarray(prim.colors.astype(np.float32)[corners])
        mat = prim.material if prim.material is not None else -1
        self.items.append(DrawItem(positions, normals, has_vn, tangents, uvs, colors, mat))
        self._bounds = None

    # -- queries --------------------------------------------------------------
    def default_material(self) -> int:
        return len(self.materials)

    def triangle_count(self) -> int:
        return sum(it.triangle_count for it in self.items)

    def bounds(self):
        if self._bounds is None and self.items:
            mn = np.min([it.positions.min(axis=0) for it in self.items], axis=0)
            mx = np.max([it.positions.max(axis=0) for it in self.items], axis=0)
            self._bounds = (mn.astype(np.float32), mx.astype(np.float32))
        return self._bounds

    def bounds_or_unit(self):
        b = self.bounds()
        if b is None:
            return (np.full(3, -0.5, np.float32), np.full(3, 0.5, np.float32))
        return b

    def lights_for(self, opts: RenderOptions) -> List[PlacedLight]:
        """Scene lights, or the options' fallback light (src/prepare.rs:1197-1204)."""
        if opts.use_scene_lights and self.scene_lights:
            return list(self.scene_lights)
        spec: LightSpec = opts.light
        az, el = math.radians(spec.azimuth_deg), math.radians(spec.elevation_deg)
        toward = _normalise([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
        return [PlacedLight(abi.PT_LIGHT_DIRECTIONAL, (1.0, 1.0, 1.0), math.pi * max(spec.intensity, 0.0),
                            (0.0, 0.0, 0.0), tuple(-toward), None, 0.0, math.pi / 4)]

    # -- ABI packing ------------------------------------------------------------
    def _binding(self, r: Optional[TextureRef]) -> abi.pt_texture_binding:
        b = abi.no_binding()
        if r is None or not (0 <= r.texture < len(self.textures)) or self.textures[r.texture] is None:
            return b
        b.texture = r.texture
        b.uv_set = r.effective_uv_set()
        t = r.transform
        if t is not None and not t.is_identity() and all(math.isfinite(v) for v in t.matrix()):
            b.has_transform = 1
            for k, v in enumerate(t.matrix()):
                b.transform[k] = v
        return b

    def _pt_material(self, m: Optional[Material]) -> abi.pt_material:
        c = abi.pt_material()
        if m is None:  # PreparedMaterial::fallback
            c.base_color[:] = (0.7, 0.7, 0.75, 1.0)
            for name in ("base_color_texture", "metallic_roughness_texture", "normal_texture", "occlusion_texture",
                         "emissive_texture"):
                setattr(c, name, abi.no_binding())
            c.metallic, c.roughness = 0.0, 1.0
            c.normal_scale, c.occlusion_strength = 1.0, 1.0
            c.alpha_mode, c.alpha_cutoff, c.ior = abi.PT_ALPHA_OPAQUE, 0.5, 1.5
            self._ext_none(c)
            return c
        ext = m.ext
        strength = max(_fin(ext.emissive_strength, 1.0), 0.0) if ext.emissive_strength is not None else 1.0
        bc = m.base_color
        c.base_color[:] = (_fin(bc[0], 1.0), _fin(bc[1], 1.0), _fin(bc[2], 1.0), _clamp(_fin(bc[3], 1.0), 0.0, 1.0))
        c.base_color_texture = self._binding(m.base_color_texture)
        c.metallic = _clamp(_fin(m.metallic, 1.0), 0.0, 1.0)
        c.roughness = _clamp(_fin(m.roughness, 1.0), 0.0, 1.0)
        c.metallic_roughness_texture = self._binding(m.metallic_roughness_texture)
        c.normal_texture = self._binding(m.normal_texture)
        c.normal_scale = _fin(m.normal_scale, 1.0)
        c.occlusion_texture = self._binding(m.occlusion_texture)
        c.occlusion_strength = _clamp(_fin(m.occlusion_strength, 1.0), 0.0, 1.0)
        e = [max(_fin(float(v), 0.0), 0.0) for v in m.emissive_factor]
        # f32 product, as the reference multiplies two f32 values.
        c.emissive[:] = [float(np.float32(np.float32(v) * np.float32(strength))) for v in e]
        c.emissive_texture = self._binding(m.emissive_texture)
        c.alpha_mode = m.alpha_mode
        c.alpha_cutoff = m.alpha_cutoff
        c.double_sided = 1 if m.double_sided else 0
        c.unlit = 1 if ext.unlit else 0
        c.ior = max(_fin(ext.ior, 1.5), 1.0) if ext.ior is not None else 1.5
        self._ext_none(c)
        flags = 0
        if ext.specular is not None:
            s = ext.specular
            flags |= abi.PT_EXT_SPECULAR
            c.specular_factor = s.factor
            c.specular_texture = self._binding(s.factor_texture)
            c.specular_color_factor[:] = s.color_factor
            c.specular_color_texture = self._binding(s.color_texture)
        if ext.transmission is not None:
            flags |= abi.PT_EXT_TRANSMISSION
            c.transmission_factor = ext.transmission.factor
            c.transmission_texture = self._binding(ext.transmission.factor_texture)
        if ext.volume is not None:
            v = ext.volume
            flags |= abi.PT_EXT_VOLUME
            c.thickness_factor = v.thickness
            c.thickness_texture = self._binding(v.thickness_texture)
            c.attenuation_distance = v.effective_attenuation_distance()
            c.attenuation_color[:] = v.attenuation_color
        if ext.clearcoat is not None:
            cc = ext.clearcoat
            flags |= abi.PT_EXT_CLEARCOAT
            c.clearcoat_factor = cc.factor
            c.clearcoat_texture = self._binding(cc.factor_texture)
            c.clearcoat_roughness_factor = cc.roughness
            c.clearcoat_roughness_texture = self._binding(cc.roughness_texture)
            c.clearcoat_normal_texture = self._binding(cc.normal_texture)
            c.clearcoat_normal_scale = cc.normal_scale
        if ext.sheen is not None:
            sh = ext.sheen
            flags |= abi.PT_EXT_SHEEN
            c.sheen_color_factor[:] = sh.color_factor
            c.sheen_color_texture = self._binding(sh.color_texture)
            c.sheen_roughness_factor = sh.roughness
            c.sheen_roughness_texture = self._binding(sh.roughness_texture)
        if ext.anisotropy is not None:
            a = ext.anisotropy
            flags |= abi.PT_EXT_ANISOTROPY
            c.anisotropy_strength = a.strength
            c.anisotropy_rotation = a.rotation
            c.anisotropy_texture = self._binding(a.texture)
        if ext.iridescence is not None:
            ir = ext.iridescence
            flags |= abi.PT_EXT_IRIDESCENCE
            c.iridescence_factor = ir.factor
            c.iridescence_texture = self._binding(ir.factor_texture)
            c.iridescence_ior = ir.ior
            c.iridescence_thickness_min = ir.thickness_min
            c.iridescence_thickness_max = ir.thickness_max
            c.iridescence_thickness_texture = self._binding(ir.thickness_texture)
        if ext.diffuse_transmission is not None:
            d = ext.diffuse_transmission
            flags |= abi.PT_EXT_DIFFUSE_TRANSMISSION
            c.diffuse_transmission_factor = d.factor
            c.diffuse_transmission_texture = self._binding(d.factor_texture)
            c.diffuse_transmission_color_factor[:] = d.color_factor
            c.diffuse_transmission_color_texture = self._binding(d.color_texture)
        if ext.dispersion is not None:
            flags |= abi.PT_EXT_DISPERSION
            c.dispersion = ext.dispersion
        c.ext_flags = flags
        return c

    @staticmethod
    def _ext_none(c: abi.pt_material) -> None:
        for name, _ in abi.pt_material._fields_:
            if name.endswith("_texture") and name not in (
                    "base_color_texture", "metallic_roughness_texture", "normal_texture", "occlusion_texture",
                    "emissive_texture"):
                setattr(c, name, abi.no_binding())
        c.specular_factor = 1.0
        c.specular_color_factor[:] = (1.0, 1.0, 1.0)
        c.attenuation_distance = math.inf
        c.attenuation_color[:] = (1.0, 1.0, 1.0)
        c.clearcoat_normal_scale = 1.0
        c.iridescence_ior = 1.3
        c.iridescence_thickness_min = 100.0
        c.iridescence_thickness_max = 400.0
        c.diffuse_transmission_color_factor[:] = (1.0, 1.0, 1.0)

    def to_desc(self, opts: Optional[RenderOptions] = None) -> "SceneDesc":
        return SceneDesc(self, opts or RenderOptions())


def _fptr(a: Optional[np.ndarray]):
    if a is None:
        return C.POINTER(C.c_float)()
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


class SceneDesc:
    """A packed `pt_scene_desc` plus the buffers it points into."""

    def __init__(self, scene: PreparedScene, opts: RenderOptions):
        self._keep = []
        items = (abi.pt_draw_item * max(len(scene.items), 1))()
        nmat = len(scene.materials) + 1
        for i, it in enumerate(scene.items):
            d = items[i]
            d.triangle_count = it.triangle_count
            d.positions = _fptr(it.positions)
            d.normals = _fptr(it.normals)
            d.has_vertex_normals = 1 if it.has_vertex_normals else 0
            d.tangents = _fptr(it.tangents)
            for s in range(abi.PT_MAX_UV_SETS):
                d.uvs[s] = _fptr(it.uvs[s] if s < len(it.uvs) else None)
            d.colors = _fptr(it.colors)
            mat = it.material
            d.material = mat if 0 <= mat < nmat - 1 else nmat - 1
            self._keep.append(it)
        mats = (abi.pt_material * nmat)()
        for i, m in enumerate(scene.materials):
            mats[i] = scene._pt_material(m)
        mats[nmat - 1] = scene._pt_material(None)
        texs = (abi.pt_texture * max(len(scene.textures), 1))()
        for i, t in enumerate(scene.textures):
            if t is None:
                continue
            if t.pixels.dtype == np.uint8:
                px = np.ascontiguousarray(t.pixels)
                texs[i].format = abi.PT_PIXELS_RGBA8
            else:
                px = np.ascontiguousarray(t.pixels, dtype=np.float32)
                texs[i].format = abi.PT_PIXELS_RGBA_F32
            self._keep.append(px)
            texs[i].width = px.shape[1]
            texs[i].height = px.shape[0]
            texs[i].pixels = px.ctypes.data
            texs[i].mag_filter = t.sampler.mag_filter
            texs[i].min_filter = t.sampler.min_filter
            texs[i].wrap_s = t.sampler.wrap_s
            texs[i].wrap_t = t.sampler.wrap_t
        lights = scene.lights_for(opts)
        lts = (abi.pt_light * max(len(lights), 1))()
        for i, L in enumerate(lights):
            lts[i].kind = L.kind
            lts[i].color[:] = L.color
            lts[i].intensity = L.intensity
            lts[i].position[:] = L.position
            lts[i].direction[:] = L.direction
            lts[i].has_range = 1 if L.range is not None else 0
            lts[i].range = L.range if L.range is not None else 0.0
            lts[i].inner_cone_angle = L.inner_cone_angle
            lts[i].outer_cone_angle = L.outer_cone_angle
        self.items, self.materials, self.textures, self.lights = items, mats, texs, lts
        self.desc = abi.pt_scene_desc(
            len(scene.items), items, nmat, mats, len(scene.textures), texs, len(lights), lts)
        self.triangle_count = scene.triangle_count()

    def ref(self):
        return C.byref(self.desc)


# ----------------------------------------------------------------------------- camera


@dataclass
class Camera:
    """Camera placement (src/camera.rs:63-91)."""

    eye: tuple
    forward: tuple
    side: tuple
    up: tuple
    half_w: float
    half_h: float
    projection: Projection = Projection.Perspective
    near: float = 0.01   # clip planes (DepthDebug): Camera::near / far
    far: float = 1000.0

    def to_c(self) -> abi.pt_camera:
        c = abi.pt_camera()
        c.eye[:] = self.eye
        c.forward[:] = self.forward
        c.side[:] = self.side
        c.up[:] = self.up
        c.half_w = self.half_w
        c.half_h = self.half_h
        c.projection = int(self.projection)
        return c

    @staticmethod
    def from_scene_camera(cam: SceneCamera, width: int, height: int, mn=None, mx=None) -> "Camera":
        """Camera::from_scene_camera (src/camera.rs:208-332); `mn` / `mx`
        bound the scene (the far plane of an infinite or unset zfar)."""
        w = cam.world
        eye = w[:3, 3]
        forward = _normalise(-w[:3, 2])
        if float(np.dot(forward, forward)) < 0.5:
            forward = np.array([0.0, 0.0, -1.0])
        up_hint = _normalise(w[:3, 1])
        side = _normalise(np.cross(forward, up_hint))
        if float(np.dot(side, side)) < 0.5:
            side = _normalise(np.cross(forward, [0.0, 1.0, 0.0]))
            if float(np.dot(side, side)) < 0.5:
                side = np.array([1.0, 0.0, 0.0])
        up = np.cross(side, forward)
        aspect = max(width, 1) / max(height, 1)
        far_extent = 0.0
        if mn is not None and mx is not None:
            for i in range(8):
                c = np.array([mx[0] if i & 1 else mn[0], mx[1] if i & 2 else mn[1], mx[2] if i & 4 else mn[2]], float)
                d = float(np.dot(c - eye, forward))
                if math.isfinite(d):
                    far_extent = max(far_extent, d)
        zfar = cam.zfar
        if cam.perspective:
            yfov = cam.yfov if (math.isfinite(cam.yfov) and 1e-4 < cam.yfov < math.pi - 1e-3) else math.pi / 3
            th = math.tan(yfov * 0.5)
            near = cam.znear if (math.isfinite(cam.znear) and cam.znear > 0.0) else 0.01
            far = zfar if (zfar is not None and math.isfinite(zfar) and zfar > near) else \
                max(far_extent * 1.05, near * 2.0 + 1e-3)
            return Camera(tuple(eye), tuple(forward), tuple(side), tuple(up), th * aspect, th, Projection.Perspective,
                          near, far)
        hh = abs(cam.ymag) if (math.isfinite(cam.ymag) and abs(cam.ymag) > 1e-6) else 1.0
        near = cam.znear if math.isfinite(cam.znear) else 0.0
        far = zfar if (zfar is not None and math.isfinite(zfar) and zfar > near) else \
            max(far_extent * 1.05, near + 1e-3)
        return Camera(tuple(eye), tuple(forward), tuple(side), tuple(up), hh * aspect, hh, Projection.Orthographic,
                      near, far)

    @staticmethod
    def build(width: int, height: int, mn, mx, opts: RenderOptions) -> "Camera":
        """Camera::build, the auto-frame / orbit camera (src/camera.rs:357-448)."""
        off = opts.camera_target_offset if all(math.isfinite(v) for v in opts.camera_target_offset) else (0, 0, 0)
        mn, mx = np.asarray(mn, float), np.asarray(mx, float)
        center = (mn + mx) * 0.5 + np.asarray(off, float)
        extent = max(float(np.max(mx - mn)), 1e-3)
        aspect = max(width, 1) / max(height, 1)
        radius = extent * 0.5 * 1.2
        fov_y = math.radians(opts.fov_deg)
        persp = opts.projection == Projection.Perspective
        auto = radius / math.tan(fov_y * 0.5) if persp else extent * 1.5
        if opts.camera is not None:
            c = opts.camera
            el, az = math.radians(c.elevation_deg), math.radians(c.azimuth_deg)
            dist = auto * c.distance
            d = np.array([math.cos(el) * math.sin(az), math.sin(el), math.cos(el) * math.cos(az)])
            eye = center + d * dist
        else:
            dist = auto
            eye = center + np.array([0.0, 0.0, auto])
        forward = _normalise(center - eye)
        side = _normalise(np.cross(forward, [0.0, 1.0, 0.0]))
        up = np.cross(side, forward)
        th = math.tan(fov_y * 0.5)
        if persp:
            hw, hh = th * aspect, th
        else:
            zoom = opts.camera.distance if (opts.camera and math.isfinite(opts.camera.distance)
                                            and opts.camera.distance > 0) else 1.0
            half = radius * zoom
            hw, hh = (half * aspect, half) if aspect >= 1.0 else (half, half / aspect)
        if persp:
            near, far = max(dist - extent, extent * 0.01), dist + extent * 2.0
        else:
            near, far = min(dist - extent * 2.0, -extent), dist + extent * 2.0
        return Camera(tuple(eye), tuple(forward), tuple(side), tuple(up), hw, hh,
                      Projection.Perspective if persp else Projection.Orthographic, near, far)

    @staticmethod
    def resolve(scene: PreparedScene, opts: RenderOptions, width: int, height: int) -> "Camera":
        """Camera::resolve (src/camera.rs:177-188)."""
        mn, mx = scene.bounds_or_unit()
        if opts.scene_camera is not None and 0 <= opts.scene_camera < len(scene.cameras):
            return Camera.from_scene_camera(scene.cameras[opts.scene_camera], width, height, mn, mx)
        return Camera.build(width, height, mn, mx, opts)
