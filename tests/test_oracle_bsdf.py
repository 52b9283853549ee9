"""Oracle pins for the BSDF: ports of src/pathtrace.rs:2954-3228.

Quadrature (360 x 180 over the sphere) against 2^16 Owen-Sobol' BSDF samples
within 2 %, albedo <= 1.01, mixture pdf a sub-density; anisotropy strength 0
is the isotropic code path bit for bit; diffuse transmission exact values;
white Lambert albedo 1 +- 1e-3.
"""
import math

import numpy as np
import pytest

U16 = None


def sobol_u(oracle, n, seed):
    return np.ascontiguousarray(oracle.sobol_owen_4d_many(n, seed)[:, :3])


def quadrature(b):
    nt, np_ = 360, 180
    th = (np.arange(nt) + 0.5) / nt * math.pi
    ph = (np.arange(np_) + 0.5) / np_ * math.pi
    T, P = np.meshgrid(th, ph, indexing="ij")
    l = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3).astype(np.float32)
    dw = (np.sin(T) * (math.pi / nt) * (math.pi / np_) * 2.0).reshape(-1)
    f, pdf = b.eval_many(l)
    return (f.astype(np.float64) * dw[:, None]).sum(0), float((pdf.astype(np.float64) * dw).sum())


def monte_carlo(oracle, b, n, seed=12345):
    u = sobol_u(oracle, n, seed)
    _, f, pdf, ok = b.sample_many(u)
    e = np.zeros(3)
    e += (f[ok] / pdf[ok, None]).astype(np.float64).sum(0) / n
    return e


V = np.array([0.6, 0.0, 0.8], np.float32)
NG = np.array([0.0, 0.0, 1.0], np.float32)


def cases(oracle):
    ms = oracle.material_sample
    out = [
        ("rough dielectric", ms(base=(0.8, 0.5, 0.2), metallic=0.0, roughness=0.8), True),
        ("glossy dielectric", ms(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.45), True),
        ("rough metal", ms(base=(0.95, 0.64, 0.54), metallic=1.0, roughness=0.6), True),
        ("half metal", ms(base=(0.9, 0.9, 0.9), metallic=0.5, roughness=0.5), True),
        ("thin transmission", ms(base=(1, 1, 1), metallic=0.0, roughness=0.5, transmission=1.0), True),
        ("volume entering", ms(base=(1, 1, 1), metallic=0.0, roughness=0.5, transmission=1.0, thickness=1.0), True),
        ("volume leaving", ms(base=(1, 1, 1), metallic=0.0, roughness=0.5, transmission=1.0, thickness=1.0,
                              normal=(0, 0, -1), clearcoat_normal=(0, 0, -1)), False),
        ("clearcoat", ms(base=(0.2, 0.3, 0.8), metallic=0.0, roughness=0.7, clearcoat=1.0,
                         clearcoat_roughness=0.4), True),
        ("sheen", ms(base=(0.3, 0.1, 0.1), metallic=0.0, roughness=0.8, sheen_color=(0.9, 0.7, 0.7),
                     sheen_roughness=0.6), True),
    ]
    return out


def extension_cases(oracle):
    ms = oracle.material_sample
    brushed = dict(base=(0.95, 0.9, 0.8), metallic=1.0, roughness=0.5, anisotropy=0.9,
                   anisotropy_direction=(1, 0, 0))
    adiel = dict(base=(0.7, 0.3, 0.2), metallic=0.0, roughness=0.45, anisotropy=0.7, anisotropy_direction=(1, 0, 0))
    dt = dict(base=(0.3, 0.6, 0.2), metallic=0.0, roughness=1.0, diffuse_transmission=0.6,
              diffuse_transmission_color=(0.9, 0.5, 0.3))
    return [
        ("brushed metal (along v)", ms(**brushed)),
        ("brushed metal (across v)", ms(**{**brushed, "anisotropy_direction": (0, 1, 0)})),
        ("anisotropic dielectric", ms(**adiel)),
        ("anisotropic thin transmission", ms(**adiel, transmission=0.8)),
        ("iridescent dielectric", ms(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.3, iridescence=1.0,
                                     iridescence_thickness=550.0)),
        ("iridescent metal", ms(base=(0.9, 0.6, 0.3), metallic=1.0, roughness=0.4, iridescence=0.8,
                                iridescence_thickness=300.0)),
        ("diffuse transmission", ms(**dt)),
        ("diffuse + specular transmission", ms(**{**dt, "roughness": 0.5}, transmission=0.3)),
    ]


def check_case(oracle, name, m, front):
    ng = NG if front else -NG
    b = oracle.Bsdf(m, V / np.linalg.norm(V), ng, front)
    eq, pdf_int = quadrature(b)
    em = monte_carlo(oracle, b, 1 << 16)
    for k in range(3):
        tol = 0.02 * max(eq[k], 0.05)
        assert abs(eq[k] - em[k]) < tol, f"{name} ch{k}: quadrature {eq[k]} vs sampled {em[k]}"
        assert eq[k] <= 1.01, f"{name} ch{k}: albedo {eq[k]}"
    assert 0.5 < pdf_int <= 1.01, f"{name}: integral of pdf = {pdf_int}"


@pytest.mark.parametrize("idx", range(9))
def test_bsdf_sampling_matches_quadrature_and_conserves_energy(oracle, idx):
    name, m, front = cases(oracle)[idx]
    check_case(oracle, name, m, front)


@pytest.mark.parametrize("idx", range(8))
def test_extension_lobes_sample_their_quadrature_and_conserve_energy(oracle, idx):
    name, m = extension_cases(oracle)[idx]
    check_case(oracle, name, m, True)


def test_anisotropy_zero_is_isotropic_and_strength_stretches(oracle):
    ms = oracle.material_sample
    v = V / np.linalg.norm(V)
    base = ms(base=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.4)
    zero = ms(base=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.4, anisotropy_direction=(1, 0, 0))
    iso, z = oracle.Bsdf(base, v, NG, True), oracle.Bsdf(zero, v, NG, True)
    r = np.array([-0.6, 0.0, 0.8], np.float32)
    nrm = lambda x: (np.array(x, np.float32) / np.linalg.norm(x)).astype(np.float32)  # noqa: E731
    for l in [r, nrm([-0.3, 0.1, 0.9]), nrm([0.2, -0.5, 0.8]), nrm([-0.8, 0.3, 0.5])]:
        fa, pa, _ = iso.eval(l)
        fb, pb, _ = z.eval(l)
        assert np.array_equal(fa, fb) and pa == pb
    lx = nrm(r + np.array([0.35, 0, 0], np.float32))
    ly = nrm(r + np.array([0, 0.35, 0], np.float32))
    ratio = lambda b: b.eval(lx)[0][0] / b.eval(ly)[0][0]  # noqa: E731
    iso_ratio = ratio(iso)
    ax = ms(base=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.4, anisotropy=0.8, anisotropy_direction=(1, 0, 0))
    ay = ms(base=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.4, anisotropy=0.8, anisotropy_direction=(0, 1, 0))
    assert ratio(oracle.Bsdf(ax, v, NG, True)) > 2.0 * iso_ratio
    assert ratio(oracle.Bsdf(ay, v, NG, True)) < 0.5 * iso_ratio
    b = oracle.Bsdf(ax, v, NG, True)
    u = sobol_u(oracle, 64, 7)
    l, f, pdf, ok = b.sample_many(u)
    for i in np.nonzero(ok)[0]:
        f2, p2, _ = b.eval(l[i])
        assert abs(pdf[i] - p2) <= 1e-4 * max(pdf[i], 1.0)
        assert np.array_equal(f[i], f2)


def test_iridescence_strength_zero_is_untouched_and_one_tints(oracle):
    ms = oracle.material_sample
    v = np.array([0.3, 0.0, 0.95], np.float32)
    v = v / np.linalg.norm(v)
    r = np.array([-0.3, 0.0, 0.95], np.float32)
    plain = ms(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.2)
    off = ms(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.2, iridescence_thickness=550.0)
    fp, pp, _ = oracle.Bsdf(plain, v, NG, True).eval(r)
    fo, po, _ = oracle.Bsdf(off, v, NG, True).eval(r)
    assert np.array_equal(fp, fo) and pp == po
    on = ms(base=(0.8, 0.8, 0.8), metallic=0.0, roughness=0.2, iridescence_thickness=550.0, iridescence=1.0)
    fi, _, _ = oracle.Bsdf(on, v, NG, True).eval(r)
    spread = lambda f: (f.max() - f.min()) / f.max()  # noqa: E731
    assert spread(fp) < 1e-3
    assert spread(fi) > 0.1


def test_diffuse_transmission_moves_lambert_energy_below_the_surface(oracle):
    ms = oracle.material_sample
    n = np.array([0, 0, 1], np.float32)
    m = ms(base=(1, 1, 1), metallic=0.0, roughness=1.0, specular=0.0, diffuse_transmission=1.0,
           diffuse_transmission_color=(0.5, 1.0, 0.25))
    b = oracle.Bsdf(m, n, n, True)
    up = np.array([0.3, 0.2, 0.9], np.float32)
    fa, pa, probs = b.eval(up / np.linalg.norm(up))
    assert np.all(fa == 0) and pa == 0.0
    l = np.array([0.3, 0.2, -0.9], np.float32)
    l = l / np.linalg.norm(l)
    fb, pb, probs = b.eval(l)
    nl = -l[2]
    for k, c in enumerate([0.5, 1.0, 0.25]):
        assert abs(fb[k] - c * nl / math.pi) < 1e-5
    assert abs(pb - nl / math.pi) < 1e-5
    assert probs[5] == 1.0
    e = monte_carlo(oracle, b, 4096)
    assert np.all(np.abs(e - np.array([0.5, 1.0, 0.25])) < 2e-3), e
    m2 = ms(base=(1, 1, 1), metallic=0.0, roughness=1.0, specular=0.0, diffuse_transmission=0.5,
            diffuse_transmission_color=(0.5, 1.0, 0.25))
    b2 = oracle.Bsdf(m2, n, n, True)
    fa, _, _ = b2.eval(np.array([0, 0, 1], np.float32))
    assert abs(fa[0] - 0.5 / math.pi) < 1e-5
    e = monte_carlo(oracle, b2, 4096)
    assert abs(e[1] - 1.0) < 2e-3 and abs(e[0] - 0.75) < 2e-3, e


def test_white_lambert_albedo_is_exact(oracle):
    m = oracle.material_sample(base=(1, 1, 1), metallic=0.0, roughness=1.0, specular=0.0)
    n = np.array([0, 0, 1], np.float32)
    e = monte_carlo(oracle, oracle.Bsdf(m, n, n, True), 4096)
    assert np.all(np.abs(e - 1.0) < 1e-3), e
