"""Frame sources over a renderer (src/source.rs): a pipeline pulls rendered
frames out of a scene without a container or decoder.

`RenderSource` mirrors the reference's still-scene source
(src/source.rs:35-131): codec parameters advertise raw RGBA video of the
options' size at 1/1 fps, the first `next_frame` renders and returns one
packed single-plane video frame (pts 0, stride = 4 * width), every later
call raises `Eof`, and the duration is one second.

`AnimatedRenderSource` is the animation-aware variant the reference leaves
for later (src/source.rs:12-17): frame k is the scene at time
start + k / fps, rendered with `opts.time` set to that time; its pts is k
in units of 1 / fps. A renderer with `render_frame` (the CUDA path
tracer) refits the resident scene's BVH when a frame keeps the previous
frame's draw items and triangle counts (new streams and tables, the tree's
structure kept, bounds recomputed on the device); otherwise every frame
re-prepares the scene it is given (with the device BVH builder a few
milliseconds for 10^5-10^6 triangles). The renderer keeps its device
accumulator and wave buffers between frames.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from fractions import Fraction
from typing import Callable, List, Optional, Tuple

import numpy as np

from .options import RenderOptions


class Eof(Exception):
    """oxideav_core::Error::Eof: the source has no more frames."""


@dataclass
class CodecParameters:
    """The video shape a source advertises (oxideav_core::CodecParameters)."""

    codec_id: str = "rawvideo"
    media_type: str = "video"
    width: Optional[int] = None
    height: Optional[int] = None
    pixel_format: str = "rgba"
    frame_rate: Tuple[int, int] = (1, 1)


@dataclass
class VideoPlane:
    stride: int
    data: bytes


@dataclass
class VideoFrame:
    pts: Optional[int]
    planes: List[VideoPlane] = field(default_factory=list)


def rgba_image_to_video_frame(img: np.ndarray, pts: int) -> VideoFrame:
    """One packed RGBA8 plane (src/source.rs:133-141)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape[:2]
    return VideoFrame(pts=pts, planes=[VideoPlane(stride=4 * w, data=img.tobytes())])


def _video_params(opts: RenderOptions, rate: Tuple[int, int]) -> CodecParameters:
    return CodecParameters(width=opts.width, height=opts.height, frame_rate=rate)


class RenderSource:
    """A still scene as a one-frame source (src/source.rs:64-131)."""

    def __init__(self, scene, renderer, opts: RenderOptions):
        self.scene = scene
        self.renderer = renderer
        self.opts = opts
        self._params = _video_params(opts, (1, 1))
        self._emitted = False

    def params(self) -> CodecParameters:
        return self._params

    def next_frame(self) -> VideoFrame:
        if self._emitted:
            raise Eof()
        img = self.renderer.render(self.scene, self.opts)
        self._emitted = True
        return rgba_image_to_video_frame(img, 0)

    def duration_micros(self) -> Optional[int]:
        return 1_000_000


class AnimatedRenderSource:
    """`frames` frames of an animated scene at `fps` (numerator,
    denominator). `scene_at(t)` returns the scene at time t (a
    PreparedScene); a static scene object may be given instead."""

    def __init__(self, scene_at, renderer, opts: RenderOptions, frames: int, fps: Tuple[int, int] = (30, 1),
                 start: float = 0.0):
        if frames < 1:
            raise ValueError("an animated source needs at least one frame")
        num, den = int(fps[0]), int(fps[1])
        if num <= 0 or den <= 0:
            raise ValueError(f"frame rate must be positive, got {fps}")
        self._scene_at: Callable = scene_at if callable(scene_at) else (lambda t, s=scene_at: s)
        self.renderer = renderer
        self.opts = opts
        self.frames = frames
        self.fps = (num, den)
        self.start = float(start)
        self._params = _video_params(opts, self.fps)
        self._next = 0

    def params(self) -> CodecParameters:
        return self._params

    def time_of(self, k: int) -> float:
        return self.start + float(Fraction(k * self.fps[1], self.fps[0]))

    def next_frame(self) -> VideoFrame:
        if self._next >= self.frames:
            raise Eof()
        k = self._next
        t = self.time_of(k)
        render = getattr(self.renderer, "render_frame", self.renderer.render)
        img = render(self._scene_at(t), self.opts.replace(time=t))
        self._next += 1
        return rgba_image_to_video_frame(img, k)

    def duration_micros(self) -> Optional[int]:
        return int(Fraction(self.frames * self.fps[1] * 1_000_000, self.fps[0]))


__all__ = ["AnimatedRenderSource", "CodecParameters", "Eof", "RenderSource", "VideoFrame", "VideoPlane",
           "rgba_image_to_video_frame"]
