"""Texture mip chains generated on the device at scene upload: the scene's
texel pool equals, bit for bit, the oracle's build_mips
(src/texture.rs:324-383) for both chains (sRGB-decoded colour and linear
data) of RGBA8 and f32 textures of odd, thin and power-of-two sizes.
Textured renders against the oracle are covered by the HDR parity tests."""
import numpy as np
import pytest

from oxideav_render_b200 import testscenes as ts
from oxideav_render_b200.scene import PreparedScene, Primitive, Texture, TextureRef

pytestmark = pytest.mark.gpu


def level_sizes(w: int, h: int):
    out = [(w, h)]
    while (w, h) != (1, 1):
        w, h = max(w // 2, 1), max(h // 2, 1)
        out.append((w, h))
    return out


def expected_pool(oracle, textures):
    parts = []
    for px in textures:
        s, lin = oracle.texture_mips(px, True), oracle.texture_mips(px, False)
        o = 0
        for w, h in level_sizes(px.shape[1], px.shape[0]):
            parts += [s[o:o + w * h], lin[o:o + w * h]]
            o += w * h
        assert o == len(s) == len(lin)
    return np.concatenate(parts)


def textured_scene(textures):
    s = PreparedScene()
    ids = [s.add_texture(Texture(px)) for px in textures]
    m = ts.diffuse_material((0.8, 0.8, 0.8), 1.0)
    m.base_color_texture = TextureRef(ids[0])
    mat = s.add_material(m)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    s.add_primitive(Primitive(tri, np.array([0, 1, 2], np.uint32), material=mat))
    return s


def test_device_mips_equal_the_oracle(ctx, oracle):
    rng = np.random.default_rng(3)
    checker = np.zeros((512, 512, 4), np.uint8)
    checker[(np.arange(512)[:, None] // 32 + np.arange(512)[None, :] // 32) % 2 == 0] = (230, 230, 230, 255)
    checker[..., 3] = 255
    textures = [rng.integers(0, 256, (23, 37, 4), dtype=np.uint8),
                rng.integers(0, 256, (1, 1, 4), dtype=np.uint8),
                (rng.random((5, 16, 4)) * 4.0).astype(np.float32),
                checker,
                rng.integers(0, 256, (1, 300, 4), dtype=np.uint8),
                rng.integers(0, 256, (129, 2, 4), dtype=np.uint8)]
    scene = textured_scene(textures)
    sid = ctx.upload(scene.to_desc(ts.pt_opts(8, 1, 1)))
    try:
        got = ctx.scene_texels(sid)
    finally:
        ctx.release(sid)
    want = expected_pool(oracle, textures)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_scene_without_textures_has_an_empty_pool(ctx):
    sid = ctx.upload(ts.lambert_plane(0.5).to_desc(ts.pt_opts(8, 1, 1)))
    try:
        assert ctx.scene_texels(sid).shape == (0, 4)
    finally:
        ctx.release(sid)
