"""Oracle pins: sampler, textures, spherical triangles, environment map.

Ports of the reference's known-answer tests: src/pathtrace.rs:2866-2908
(Sobol' published points, Owen stratification), :3232-3342 (spherical
triangles, environment pdf), src/texture.rs:1059-1140 (wrap modes, bilinear,
sRGB decode, mip chains).
"""
import math

import numpy as np
import pytest

from oxideav_render_b200 import abi
from oxideav_render_b200.scene import Sampler


def to_unit(v: int) -> float:
    return (v >> 8) * (1.0 / 16777216.0)


def test_sobol_unscrambled_dims_match_published_points(oracle):
    lib = oracle.lib()
    table = [
        [0.0, 0.0, 0.0, 0.0], [0.5, 0.5, 0.5, 0.5], [0.75, 0.25, 0.25, 0.25], [0.25, 0.75, 0.75, 0.75],
        [0.375, 0.375, 0.625, 0.875], [0.875, 0.875, 0.125, 0.375], [0.625, 0.125, 0.875, 0.625],
        [0.125, 0.625, 0.375, 0.125],
    ]
    for i, row in enumerate(table):
        g = i ^ (i >> 1)
        got = [to_unit(lib.oracle_sobol(g, d)) for d in range(4)]
        assert got == row, f"point {i}"
    cells = np.zeros(16, int)
    for i in range(16):
        x = int(to_unit(lib.oracle_sobol(i, 0)) * 4)
        y = int(to_unit(lib.oracle_sobol(i, 1)) * 4)
        cells[y * 4 + x] += 1
    assert np.all(cells == 1), cells


def test_owen_scrambling_preserves_stratification(oracle):
    for seed in [1, 77, 0xDEADBEEF]:
        cells = np.zeros(64, int)
        for i in range(64):
            p = oracle.sobol_owen_4d(i, seed)
            cells[int(p[0] * 8) * 8 + int(p[1] * 8)] += 1
            assert np.all((p >= 0) & (p < 1))
        assert np.all(cells == 1), seed


def test_pcg_hash_known_values(oracle):
    # state = x*747796405 + 2891336453; RXS-M-XS output permutation.
    def pcg(x):
        s = (x * 747796405 + 2891336453) & 0xFFFFFFFF
        w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
        return ((w >> 22) ^ w) & 0xFFFFFFFF
    for x in [0, 1, 2, 12345, 0xFFFFFFFF, 0x80000000]:
        assert oracle.lib().oracle_pcg_hash(x) == pcg(x)


# ----------------------------------------------------------------------------- textures

TWO_BY_ONE = np.array([[[0, 0, 0, 255], [255, 255, 255, 255]]], np.uint8)


def test_nearest_and_wrap_modes(oracle):
    near = Sampler(abi.PT_FILTER_NEAREST, abi.PT_MIN_NEAREST)
    s = lambda u, smp: oracle.texture_sample(TWO_BY_ONE, smp, u, 0.5, 0.0, False)[0][0]  # noqa: E731
    assert s(0.25, near) == 0.0
    assert s(0.75, near) == 1.0
    assert s(1.25, near) == 0.0, "repeat"
    clamp = Sampler(abi.PT_FILTER_NEAREST, abi.PT_MIN_NEAREST, abi.PT_WRAP_CLAMP, abi.PT_WRAP_CLAMP)
    assert s(1.25, clamp) == 1.0
    assert s(-3.0, clamp) == 0.0
    mirror = Sampler(abi.PT_FILTER_NEAREST, abi.PT_MIN_NEAREST, abi.PT_WRAP_MIRROR, abi.PT_WRAP_REPEAT)
    assert s(1.25, mirror) == 1.0
    assert s(1.75, mirror) == 0.0


def test_bilinear_midpoint_and_srgb_decode(oracle):
    clamp = Sampler(wrap_s=abi.PT_WRAP_CLAMP, wrap_t=abi.PT_WRAP_CLAMP)
    mid = oracle.texture_sample(TWO_BY_ONE, clamp, 0.5, 0.5, 0.0, False)[0][0]
    assert abs(mid - 0.5) < 1e-6
    g = np.array([[[128, 128, 128, 255]]], np.uint8)
    v = oracle.texture_sample(g, Sampler(), 0.3, 0.3, 0.0, True)[0][0]
    assert abs(v - 0.2158) < 1e-3
    lin = oracle.texture_sample(g, Sampler(), 0.3, 0.3, 0.0, False)[0][0]
    assert abs(lin - 128.0 / 255.0) < 1e-6


def test_mip_chain_box_filters_to_mean(oracle):
    px = np.zeros((4, 4, 4), np.uint8)
    for y in range(4):
        for x in range(4):
            v = 255 if (x + y) % 2 == 0 else 0
            px[y, x] = (v, v, v, 255)
    _, levels, top = oracle.texture_sample(px, Sampler(), 0.1, 0.1, 0.0, False)
    assert levels == 3
    assert abs(top[0] - 0.5) < 1e-6
    # A large level of detail selects the top level (trilinear default).
    v = oracle.texture_sample(px, Sampler(), 0.1, 0.1, math.log2(40.0), False)[0]
    assert abs(v[0] - 0.5) < 1e-5
    # Level 0 with bilinear magnification at an exact texel centre.
    v0 = oracle.texture_sample(px, Sampler(), 0.125, 0.125, 0.0, False)[0]
    assert abs(v0[0] - 1.0) < 1e-6


def test_non_power_of_two_mips_terminate(oracle):
    px = np.full((3, 5, 4), 255, np.uint8)
    _, levels, top = oracle.texture_sample(px, Sampler(), 0.5, 0.5, 0.0, True)
    assert levels == 3  # 5x3 -> 2x1 -> 1x1
    assert abs(top[0] - 1.0) < 1e-6


# ----------------------------------------------------------------------------- spherical triangles


def test_octant_triangle_subtends_half_pi(oracle):
    f = lambda *v: np.array(v, np.float32).ctypes.data_as(oracle.C.POINTER(oracle.C.c_float))  # noqa: E731
    o = oracle.lib().oracle_triangle_solid_angle(f(0, 0, 0), f(1, 0, 0), f(0, 1, 0), f(0, 0, 1))
    assert abs(o - math.pi / 2) < 1e-5


def test_spherical_triangle_samples_are_uniform_in_solid_angle(oracle):
    C = oracle.C
    p = np.array([0.1, -0.2, 0.0], np.float32)
    a, b, c = (np.array(v, np.float32) for v in ([-0.6, 0.3, 1.0], [1.2, -0.4, 0.8], [0.2, 1.1, 1.4]))
    ptr = lambda x: x.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    omega = oracle.lib().oracle_triangle_solid_angle(ptr(p), ptr(a), ptr(b), ptr(c))
    n = np.cross(b - a, c - a).astype(np.float64)
    g = lambda d: (d[..., 0] + 0.3) ** 2 + d[..., 1]  # noqa: E731
    steps = 600
    i, j = np.meshgrid(np.arange(steps), np.arange(steps), indexing="ij")
    keep = j < steps - i
    u = (i[keep] + 1.0 / 3.0) / steps
    v = (j[keep] + 1.0 / 3.0) / steps
    q = a + (b - a) * u[:, None] + (c - a) * v[:, None]
    to = q - p
    r2 = np.sum(to * to, axis=1)
    d = to / np.sqrt(r2)[:, None]
    nn = n / np.linalg.norm(n)
    dw = np.abs(d @ nn) / r2
    expect = float(np.sum(g(d) * dw) / np.sum(dw))
    area2 = np.linalg.norm(n)
    assert abs(np.sum(dw) * 0.5 * area2 / steps ** 2 * 2.0 / omega - 1.0) < 0.02
    m = 1 << 15
    us = oracle.sobol_owen_4d_many(m, 5)
    out = np.zeros(3, np.float32)
    vals = np.zeros((m, 3))
    for k in range(m):
        ok = oracle.lib().oracle_sample_spherical_triangle(ptr(p), ptr(a), ptr(b), ptr(c), float(us[k, 0]),
                                                          float(us[k, 1]), ptr(out))
        assert ok
        vals[k] = out
    got = float(np.mean(g(vals)))
    assert abs(got - expect) < 0.01 * max(abs(expect), 0.1), (got, expect)
    # Every direction hits the triangle.
    t = ((a - p) @ n) / (vals @ n)
    hit = p + vals * t[:, None]
    e1, e2, r = b - a, c - a, hit - a
    d11, d12, d22 = e1 @ e1, e1 @ e2, e2 @ e2
    r1, r2_ = r @ e1, r @ e2
    det = d11 * d22 - d12 * d12
    bu = (d22 * r1 - d12 * r2_) / det
    bv = (d11 * r2_ - d12 * r1) / det
    assert np.all(1 - bu - bv > -1e-3) and np.all(bu > -1e-3) and np.all(bv > -1e-3)


# ----------------------------------------------------------------------------- environment


def test_environment_pdf_is_normalised_and_matches_samples(oracle):
    w, h = 32, 16
    img = np.zeros((h, w, 4), np.float32)
    img[...] = (0.1, 0.1, 0.1, 1.0)
    img[3:5, 20:23, :3] = (50.0, 40.0, 30.0)
    env = oracle.OracleEnv(img, 1.0)
    n = 400
    th = (np.arange(n) + 0.5) / n * math.pi
    ph = (np.arange(2 * n) + 0.5) / (2 * n) * 2 * math.pi
    total = 0.0
    for t in th:
        for p_ in ph:
            d = np.array([math.sin(t) * math.cos(p_), math.cos(t), math.sin(t) * math.sin(p_)], np.float32)
            total += env.pdf(d) * math.sin(t) * (math.pi / n) * (math.pi / n)
    assert abs(total - 1.0) < 0.01, total
    sun = 0
    for i in range(1000):
        u = oracle.sobol_owen_4d(i, 9)
        d, le, pdf = env.sample(float(u[0]), float(u[1]))
        assert abs(pdf - env.pdf(d)) <= 1e-3 * max(pdf, 1.0)
        sun += le[0] > 10.0
    assert sun > 800, sun


def test_dispersion_iors_spread_around_the_centre_index(oracle):
    C = oracle.C
    out = np.zeros(3, np.float32)
    p = out.ctypes.data_as(C.POINTER(C.c_float))
    oracle.lib().oracle_dispersion_iors(1.5, 0.0, p)
    assert list(out) == [1.5, 1.5, 1.5]
    oracle.lib().oracle_dispersion_iors(1.5, 0.36, p)
    assert out[0] < out[1] < out[2]
    assert abs(out[2] - out[0] - 0.5 * 0.05 * 0.36) < 1e-6
    oracle.lib().oracle_dispersion_iors(1.01, 100.0, p)
    assert np.all(out >= 1.0)


def test_iridescent_fresnel_is_bounded_coloured_and_fades(oracle):
    C = oracle.C

    def irid(outside, film, f0, thick, cos):
        f0a = np.array(f0, np.float32)
        out = np.zeros(3, np.float32)
        oracle.lib().oracle_iridescent_fresnel(outside, film, f0a.ctypes.data_as(C.POINTER(C.c_float)), thick, cos,
                                               out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    spread = lambda f: float(f.max() - f.min())  # noqa: E731
    f = irid(1.0, 1.3, [0.04] * 3, 400.0, 1.0)
    assert np.all((f >= 0) & (f <= 1))
    assert spread(f) > 0.02
    g = irid(1.0, 1.3, [0.04] * 3, 401.0, 1.0)
    assert np.all(np.abs(f - g) < 0.02)
    assert spread(irid(1.0, 1.3, [0.04] * 3, 20000.0, 1.0)) < 2e-3
    assert np.all(irid(1.0, 1.3, [0.04] * 3, 400.0, 0.0) > 0.95)
    assert list(irid(1.5, 1.0, [0.04] * 3, 400.0, 0.1)) == [1.0, 1.0, 1.0]
