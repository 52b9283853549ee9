"""Render options mirroring oxideav-render's options surface.

`RenderOptions`, `PathTraceOptions`, `LightStrategy`, `ToneMap`,
`Projection`, `LightSpec`, `CameraSpec` and `BackgroundColor` follow
src/options.rs (:13-146, :150-414, defaults :579-607) field for field, with
the same defaults and the same `validate()` rules (:643-757), so a caller of
the reference's `RenderOptions` finds the same knobs here.
"""
from __future__ import annotations

import dataclasses
import enum
import math
from dataclasses import dataclass, field
from typing import Optional

from . import abi


class RenderBackend(enum.Enum):
    """src/options.rs:13-44, plus the CUDA path tracer this library adds."""

    Scanline = "scanline"
    Raycast = "raycast"
    PathTrace = "pathtrace"
    PathTraceCuda = "pathtrace-cuda"


class LightStrategy(enum.IntEnum):
    """src/options.rs:51-64."""

    Mis = abi.PT_MIS
    LightOnly = abi.PT_LIGHT_ONLY
    BsdfOnly = abi.PT_BSDF_ONLY


class ToneMap(enum.IntEnum):
    """src/hdr.rs:28-39."""

    Clamp = abi.PT_TONE_CLAMP
    Reinhard = abi.PT_TONE_REINHARD
    AcesFitted = abi.PT_TONE_ACES


class Projection(enum.IntEnum):
    """src/options.rs:187-196."""

    Perspective = abi.PT_PERSPECTIVE
    Orthographic = abi.PT_ORTHOGRAPHIC


class ShadingMode(enum.Enum):
    """src/options.rs:150-185 (ignored by the path tracer)."""

    Flat = 0
    Gouraud = 1
    Phong = 2
    Wireframe = 3
    NormalDebug = 4
    DepthDebug = 5
    Pbr = 6


@dataclass(frozen=True)
class BackgroundColor:
    """RGBA8 clear colour (src/options.rs:198-206); default transparent black."""

    rgba: tuple = (0, 0, 0, 0)


@dataclass(frozen=True)
class LightSpec:
    """Fallback directional light (src/options.rs:208-270)."""

    azimuth_deg: float = 45.0
    elevation_deg: float = 45.0
    intensity: float = 1.0


@dataclass(frozen=True)
class CameraSpec:
    """Orbit camera override (src/options.rs:272-318)."""

    elevation_deg: float
    azimuth_deg: float
    distance: float


@dataclass(frozen=True)
class PathTraceOptions:
    """src/options.rs:67-146."""

    samples_per_pixel: int = 64
    max_bounces: int = 8
    rr_start: int = 3
    clamp: float = 0.0
    seed: int = 0
    strategy: LightStrategy = LightStrategy.Mis

    def to_c(self) -> abi.pt_path_trace_options:
        o = abi.pt_path_trace_options()
        o.samples_per_pixel = int(self.samples_per_pixel)
        o.max_bounces = int(self.max_bounces)
        o.rr_start = int(self.rr_start)
        o.clamp = float(self.clamp)
        o.seed = int(self.seed) & 0xFFFFFFFF
        o.strategy = int(self.strategy)
        return o


class InvalidOptions(ValueError):
    """oxideav_render::Error::InvalidOptions."""


@dataclass(frozen=True)
class RenderOptions:
    """src/options.rs:325-414 with the defaults of :579-607."""

    width: int = 512
    height: int = 512
    background: BackgroundColor = BackgroundColor()
    shading: ShadingMode = ShadingMode.Phong
    projection: Projection = Projection.Perspective
    fov_deg: float = 60.0
    light: LightSpec = LightSpec()
    camera: Optional[CameraSpec] = None
    camera_target_offset: tuple = (0.0, 0.0, 0.0)
    aa: int = 1
    tone_map: ToneMap = ToneMap.Clamp
    exposure: float = 1.0
    time: Optional[float] = None
    animation: Optional[int] = None
    scene_camera: Optional[int] = None
    use_scene_lights: bool = True
    ambient: float = 0.2
    shadows: bool = False
    shadow_map_size: int = 1024
    material_variant: Optional[int] = None
    max_ray_depth: int = 4
    reflection_roughness_cutoff: float = 0.5
    path_trace: PathTraceOptions = field(default_factory=PathTraceOptions)

    def replace(self, **kw) -> "RenderOptions":
        return dataclasses.replace(self, **kw)

    def to_c(self) -> abi.pt_render_options:
        o = abi.pt_render_options()
        o.width = max(int(self.width), 1)
        o.height = max(int(self.height), 1)
        for k in range(4):
            o.background[k] = int(self.background.rgba[k]) & 0xFF
        o.tone_map = int(self.tone_map)
        o.exposure = float(self.exposure)
        o.ambient = float(self.ambient)
        o.path_trace = self.path_trace.to_c()
        return o

    def to_raycast_c(self, near_plane: float, far_plane: float) -> abi.pt_raycast_options:
        """The raycast backend's options (include/pt_b200.h pt_raycast_options)."""
        o = abi.pt_raycast_options()
        o.width = max(int(self.width), 1)
        o.height = max(int(self.height), 1)
        o.aa = int(self.aa)
        o.shading = int(self.shading.value)
        o.light_azimuth_deg = float(self.light.azimuth_deg)
        o.light_elevation_deg = float(self.light.elevation_deg)
        o.light_intensity = float(self.light.intensity)
        for k in range(4):
            o.background[k] = int(self.background.rgba[k]) & 0xFF
        o.tone_map = int(self.tone_map)
        o.exposure = float(self.exposure)
        o.max_ray_depth = int(self.max_ray_depth)
        o.near_plane = float(near_plane)
        o.far_plane = float(far_plane)
        o.ambient = float(self.ambient)
        o.shadows = 1 if self.shadows else 0
        o.reflection_roughness_cutoff = float(self.reflection_roughness_cutoff)
        return o

    def validate(self) -> None:
        """RenderOptions::validate (src/options.rs:643-757)."""

        def bad(msg):
            raise InvalidOptions(msg)

        if self.width == 0:
            bad(f"width must be >= 1, got {self.width}")
        if self.height == 0:
            bad(f"height must be >= 1, got {self.height}")
        if not math.isfinite(self.fov_deg):
            bad(f"fov_deg must be finite, got {self.fov_deg}")
        if not (0.0 < self.fov_deg < 180.0):
            bad(f"fov_deg must be in (0, 180), got {self.fov_deg}")
        if not (1 <= self.aa <= 8):
            bad(f"aa must be in 1..=8, got {self.aa}")
        if not math.isfinite(self.light.intensity) or self.light.intensity < 0.0:
            bad(f"light.intensity must be finite and >= 0.0, got {self.light.intensity}")
        if not (math.isfinite(self.light.azimuth_deg) and math.isfinite(self.light.elevation_deg)):
            bad("light.azimuth_deg / light.elevation_deg must be finite")
        if not all(math.isfinite(v) for v in self.camera_target_offset):
            bad(f"camera_target_offset must be finite, got {self.camera_target_offset}")
        if not math.isfinite(self.exposure) or self.exposure < 0.0:
            bad(f"exposure must be finite and >= 0.0, got {self.exposure}")
        if not math.isfinite(self.ambient) or self.ambient < 0.0:
            bad(f"ambient must be finite and >= 0.0, got {self.ambient}")
        if self.time is not None and not math.isfinite(self.time):
            bad(f"time must be finite, got {self.time}")
        if not (0.0 <= self.reflection_roughness_cutoff <= 1.0):
            bad(f"reflection_roughness_cutoff must be in [0, 1], got {self.reflection_roughness_cutoff}")
        if not (16 <= self.shadow_map_size <= 8192):
            bad(f"shadow_map_size must be in 16..=8192, got {self.shadow_map_size}")
        pt = self.path_trace
        if not (1 <= pt.samples_per_pixel <= (1 << 20)):
            bad(f"path_trace.samples_per_pixel must be in 1..=1048576, got {pt.samples_per_pixel}")
        if pt.max_bounces > 1024:
            bad(f"path_trace.max_bounces must be <= 1024, got {pt.max_bounces}")
        if not math.isfinite(pt.clamp) or pt.clamp < 0.0:
            bad(f"path_trace.clamp must be finite and >= 0.0, got {pt.clamp}")
        if self.camera is not None:
            c = self.camera
            if not (math.isfinite(c.azimuth_deg) and math.isfinite(c.elevation_deg)):
                bad("camera.azimuth_deg / camera.elevation_deg must be finite")
            if not math.isfinite(c.distance) or c.distance <= 0.0:
                bad(f"camera.distance must be finite and > 0, got {c.distance}")


def radiance_key(o: RenderOptions) -> RenderOptions:
    """Options with every display-only field normalised away
    (radiance_key, src/pathtrace.rs:2402-2418)."""
    d = RenderOptions()
    return dataclasses.replace(
        o,
        background=d.background,
        shading=d.shading,
        aa=d.aa,
        tone_map=d.tone_map,
        exposure=d.exposure,
        shadows=d.shadows,
        shadow_map_size=d.shadow_map_size,
        path_trace=dataclasses.replace(o.path_trace, samples_per_pixel=d.path_trace.samples_per_pixel),
    )
