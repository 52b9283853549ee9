"""RenderSource / AnimatedRenderSource logic (ports of the reference's
src/source.rs tests :176-313) with a stand-in renderer: advertised video
parameters, one frame then Eof (idempotent), plane stride and size, one
second of duration, width / height round trip; the animated variant's
per-frame times, pts and duration. The GPU-backed renders are in
test_gpu_source.py."""
import numpy as np
import pytest

from oxideav_render_b200.options import RenderOptions
from oxideav_render_b200.source import AnimatedRenderSource, Eof, RenderSource


class PaintRenderer:
    """Paints a w x h RGBA8 image whose red channel is the frame counter."""

    def __init__(self):
        self.calls = []

    def render(self, scene, opts):
        self.calls.append((scene, opts))
        img = np.full((opts.height, opts.width, 4), 255, np.uint8)
        img[0, 0] = (len(self.calls) % 256, 0, 0, 255)
        return img


def opts(w=32, h=32):
    return RenderOptions(width=w, height=h)


def test_params_advertise_expected_video_shape():
    p = RenderSource("scene", PaintRenderer(), opts()).params()
    assert (p.codec_id, p.media_type, p.width, p.height, p.pixel_format, p.frame_rate) == \
        ("rawvideo", "video", 32, 32, "rgba", (1, 1))


def test_first_next_frame_yields_video_then_eof():
    r = PaintRenderer()
    src = RenderSource("scene", r, opts())
    f = src.next_frame()
    assert f.pts == 0 and len(f.planes) == 1
    assert f.planes[0].stride == 32 * 4 and len(f.planes[0].data) == 32 * 32 * 4
    for _ in range(2):
        with pytest.raises(Eof):
            src.next_frame()
    assert len(r.calls) == 1


def test_duration_and_dimensions_round_trip():
    src = RenderSource("scene", PaintRenderer(), opts(48, 24))
    assert src.duration_micros() == 1_000_000
    assert (src.params().width, src.params().height) == (48, 24)
    f = src.next_frame()
    assert f.planes[0].stride == 48 * 4 and len(f.planes[0].data) == 48 * 24 * 4


def test_animated_source_advances_time_per_frame():
    r = PaintRenderer()
    seen = []
    src = AnimatedRenderSource(lambda t: seen.append(t) or ("scene", t), r, opts(16, 8), frames=3, fps=(24, 1),
                               start=0.5)
    assert src.params().frame_rate == (24, 1) and src.duration_micros() == 125_000
    frames = [src.next_frame() for _ in range(3)]
    assert [f.pts for f in frames] == [0, 1, 2]
    assert seen == [0.5, 0.5 + 1 / 24, 0.5 + 2 / 24]
    assert [o.time for _, o in r.calls] == seen
    with pytest.raises(Eof):
        src.next_frame()
    # A static scene object is accepted as well.
    s2 = AnimatedRenderSource("static", PaintRenderer(), opts(), frames=1, fps=(30000, 1001))
    assert s2.duration_micros() == 33_366
    assert s2.next_frame().pts == 0


def test_animated_source_rejects_bad_shapes():
    with pytest.raises(ValueError):
        AnimatedRenderSource("s", PaintRenderer(), opts(), frames=0)
    with pytest.raises(ValueError):
        AnimatedRenderSource("s", PaintRenderer(), opts(), frames=2, fps=(0, 1))
