"""ctypes front of the oracle (oracle/_build/liboracle.so).

ORACLE — test infrastructure only: imported by tests/, by
``__graft_entry__.smoke()`` and by the bench's ``cpu_baseline`` leg, always as
the checker / the timed CPU baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(LIB_PATH)
            vp, u32, f32, i32 = C.c_void_p, C.c_uint32, C.c_float, C.c_int
            fp, dp, u32p, u8p, u64p = (C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint8), C.POINTER(C.c_uint64))
            sig = {
                "oracle_scene_create": (vp, [vp]),
                "oracle_scene_destroy": (None, [vp]),
                "oracle_scene_triangles": (C.c_uint64, [vp]),
                "oracle_env_create": (vp, [vp]),
                "oracle_env_destroy": (None, [vp]),
                "oracle_refine": (i32, [vp, vp, vp, vp, u32, u32, i32, dp, u64p]),
                "oracle_sample": (i32, [vp, vp, vp, vp, u32, u32, u32, fp]),
                "oracle_refine_rows": (i32, [vp, vp, vp, vp, u32, u32, u32, u32, u32, i32, dp, u64p]),
                "oracle_resolve_hdr": (None, [dp, u32, vp, fp]),
                "oracle_resolve_image": (None, [dp, u32, vp, u8p]),
                "oracle_primary_hits": (None, [vp, vp, vp, u32, u32p, fp, fp]),
                "oracle_closest_hit": (i32, [vp, fp, fp, f32, f32, u32p, fp, fp, C.POINTER(C.c_int)]),
                "oracle_occluded": (i32, [vp, fp, fp, f32, f32]),
                "oracle_surface": (None, [vp, u32, fp, fp, fp, fp]),
                "oracle_material_base": (None, [vp, u32, fp, fp]),
                "oracle_texture_sample": (None, [vp, f32, f32, f32, i32, fp, u32p, fp]),
                "oracle_texture_mips": (C.c_uint64, [vp, i32, fp, C.c_uint64]),
                "oracle_raycast": (i32, [vp, vp, vp, fp, C.POINTER(C.c_uint8)]),
                "oracle_emissive_table": (None, [vp, u32p, C.POINTER(u32p), C.POINTER(fp), C.POINTER(fp)]),
                "oracle_sobol_owen_4d": (None, [u32, u32, fp]),
                "oracle_sobol": (u32, [u32, u32]),
                "oracle_sampler_pattern": (None, [u32, u32, u32, u32, u32, fp]),
                "oracle_sampler_coin": (f32, [u32, u32, u32, u32, u32, u32]),
                "oracle_pcg_hash": (u32, [u32]),
                "oracle_triangle_solid_angle": (f32, [fp, fp, fp, fp]),
                "oracle_sample_spherical_triangle": (i32, [fp, fp, fp, fp, f32, f32, fp]),
                "oracle_iridescent_fresnel": (None, [f32, f32, fp, f32, f32, fp]),
                "oracle_dispersion_iors": (None, [f32, f32, fp]),
                "oracle_sheen_lut": (fp, []),
                "oracle_env_pdf": (f32, [vp, fp]),
                "oracle_env_sample": (i32, [vp, f32, f32, fp, fp, fp]),
                "oracle_bsdf_eval": (None, [fp, fp, fp, i32, fp, fp, fp, fp]),
                "oracle_bsdf_eval_many": (None, [fp, fp, fp, i32, u32, fp, fp, fp]),
                "oracle_bsdf_sample_many": (None, [fp, fp, fp, i32, u32, fp, fp, fp, fp, u8p]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def fa(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


class OracleScene:
    """The oracle's TraceScene + EmissiveLights built from a pt_scene_desc."""

    def __init__(self, desc):
        self._desc = desc
        self.ptr = lib().oracle_scene_create(C.addressof(desc.desc))
        if not self.ptr:
            raise RuntimeError("oracle_scene_create failed")

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.oracle_scene_destroy(self.ptr)
            self.ptr = None

    @property
    def triangle_count(self) -> int:
        return int(lib().oracle_scene_triangles(self.ptr))


class OracleEnv:
    def __init__(self, pixels: np.ndarray, intensity: float = 1.0):
        from_abi = _abi()
        self.pixels = np.ascontiguousarray(pixels, dtype=np.float32)
        e = from_abi.pt_environment(self.pixels.shape[1], self.pixels.shape[0],
                                    self.pixels.ctypes.data_as(C.POINTER(C.c_float)), intensity)
        self._e = e
        self.ptr = lib().oracle_env_create(C.addressof(e))

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.oracle_env_destroy(self.ptr)
            self.ptr = None

    def pdf(self, d) -> float:
        _, p = fa(d)
        return float(lib().oracle_env_pdf(self.ptr, p))

    def sample(self, u0, u1):
        d = np.zeros(3, np.float32)
        le = np.zeros(3, np.float32)
        pdf = C.c_float()
        ok = lib().oracle_env_sample(self.ptr, u0, u1, d.ctypes.data_as(C.POINTER(C.c_float)),
                                     le.ctypes.data_as(C.POINTER(C.c_float)), C.byref(pdf))
        return (d, le, pdf.value) if ok else None


_abi_mod = None


def _abi():
    global _abi_mod
    if _abi_mod is None:
        import sys
        _abi_mod = sys.modules["oxideav_render_b200.abi"]
    return _abi_mod


class OracleTracer:
    """PathTracer restated on the CPU: f64 accumulator, 4-row bands."""

    def __init__(self, scene: OracleScene, camera, opts, env: OracleEnv = None, threads: int = 0):
        self.scene, self.env = scene, env
        self.cam = camera.to_c() if hasattr(camera, "to_c") else camera
        self.opts = opts.to_c() if hasattr(opts, "to_c") else opts
        self.w, self.h = self.opts.width, self.opts.height
        self.accum = np.zeros((self.h, self.w, 4), np.float64)
        self.samples = 0
        self.threads = threads
        self.rays = np.zeros(2, np.uint64)

    def refine(self, n: int) -> None:
        if n == 0:
            return
        rc = np.zeros(2, np.uint64)
        lib().oracle_refine(self.scene.ptr, self.env.ptr if self.env else None, C.byref(self.cam),
                            C.byref(self.opts), self.samples, n, self.threads,
                            self.accum.ctypes.data_as(C.POINTER(C.c_double)),
                            rc.ctypes.data_as(C.POINTER(C.c_uint64)))
        self.rays = rc
        self.samples += n

    def hdr(self) -> np.ndarray:
        out = np.zeros((self.h, self.w, 4), np.float32)
        lib().oracle_resolve_hdr(self.accum.ctypes.data_as(C.POINTER(C.c_double)), self.samples, C.byref(self.opts),
                                 out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def image(self) -> np.ndarray:
        out = np.zeros((self.h, self.w, 4), np.uint8)
        lib().oracle_resolve_image(self.accum.ctypes.data_as(C.POINTER(C.c_double)), self.samples,
                                   C.byref(self.opts), out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    def primary_hits(self, index: int = 0):
        g = np.zeros((self.h, self.w), np.uint32)
        t = np.zeros((self.h, self.w), np.float32)
        b = np.zeros((self.h, self.w, 3), np.float32)
        lib().oracle_primary_hits(self.scene.ptr, C.byref(self.cam), C.byref(self.opts), index,
                                  g.ctypes.data_as(C.POINTER(C.c_uint32)), t.ctypes.data_as(C.POINTER(C.c_float)),
                                  b.ctypes.data_as(C.POINTER(C.c_float)))
        return g, t, b


def refine_rows(scene: OracleScene, camera, opts, env, row0: int, stride: int, count: int, first: int, samples: int,
                threads: int = 0):
    """refine() over rows row0 + i*stride (i < count) of the full frame.
    Returns (accum[count, width, 4] f64, (extension rays, shadow rays))."""
    cam = camera.to_c() if hasattr(camera, "to_c") else camera
    o = opts.to_c() if hasattr(opts, "to_c") else opts
    acc = np.zeros((count, o.width, 4), np.float64)
    rc = np.zeros(2, np.uint64)
    lib().oracle_refine_rows(scene.ptr, env.ptr if env else None, C.byref(cam), C.byref(o), row0, stride, count,
                             first, samples, threads, acc.ctypes.data_as(C.POINTER(C.c_double)),
                             rc.ctypes.data_as(C.POINTER(C.c_uint64)))
    return acc, (int(rc[0]), int(rc[1]))


def render_hdr(desc, camera, opts, env=None, threads=0):
    sc = OracleScene(desc)
    tr = OracleTracer(sc, camera, opts, env, threads)
    tr.refine(max(opts.path_trace.samples_per_pixel, 1))
    return tr.hdr()


# MaterialSample packing for the BSDF entry points (layout in oracle_integrator.cpp).
MS_FIELDS = 36


def material_sample(base=(1, 1, 1), metallic=1.0, roughness=1.0, normal=(0, 0, 1), specular=1.0,
                    specular_color=(1, 1, 1), transmission=0.0, thickness=0.0, ior=1.5, clearcoat=0.0,
                    clearcoat_roughness=0.0, clearcoat_normal=(0, 0, 1), sheen_color=(0, 0, 0),
                    sheen_roughness=0.0, anisotropy=0.0, anisotropy_direction=(0, 0, 0), iridescence=0.0,
                    iridescence_ior=1.3, iridescence_thickness=400.0, diffuse_transmission=0.0,
                    diffuse_transmission_color=(1, 1, 1), alpha=1.0) -> np.ndarray:
    a = np.zeros(MS_FIELDS, np.float32)
    a[0:3], a[3] = base, alpha
    a[4], a[5] = metallic, roughness
    a[6:9] = normal
    a[9] = specular
    a[10:13] = specular_color
    a[13], a[14], a[15] = transmission, thickness, ior
    a[16], a[17] = clearcoat, clearcoat_roughness
    a[18:21] = clearcoat_normal
    a[21:24] = sheen_color
    a[24], a[25] = sheen_roughness, anisotropy
    a[26:29] = anisotropy_direction
    a[29], a[30], a[31] = iridescence, iridescence_ior, iridescence_thickness
    a[32] = diffuse_transmission
    a[33:36] = diffuse_transmission_color
    return a


class Bsdf:
    def __init__(self, ms: np.ndarray, v, ng, front: bool):
        self.ms, self.pms = fa(ms)
        self.v, self.pv = fa(v)
        self.ng, self.png = fa(ng)
        self.front = 1 if front else 0

    def eval(self, l):
        _, pl = fa(l)
        f = np.zeros(3, np.float32)
        pdf = np.zeros(1, np.float32)
        probs = np.zeros(6, np.float32)
        lib().oracle_bsdf_eval(self.pms, self.pv, self.png, self.front, pl, f.ctypes.data_as(C.POINTER(C.c_float)),
                               pdf.ctypes.data_as(C.POINTER(C.c_float)), probs.ctypes.data_as(C.POINTER(C.c_float)))
        return f, float(pdf[0]), probs

    def eval_many(self, ls: np.ndarray):
        ls, pl = fa(ls)
        n = ls.shape[0]
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        lib().oracle_bsdf_eval_many(self.pms, self.pv, self.png, self.front, n, pl,
                                    f.ctypes.data_as(C.POINTER(C.c_float)), pdf.ctypes.data_as(C.POINTER(C.c_float)))
        return f, pdf

    def sample_many(self, u: np.ndarray):
        u, pu = fa(u)
        n = u.shape[0]
        l = np.zeros((n, 3), np.float32)
        f = np.zeros((n, 3), np.float32)
        pdf = np.zeros(n, np.float32)
        ok = np.zeros(n, np.uint8)
        lib().oracle_bsdf_sample_many(self.pms, self.pv, self.png, self.front, n, pu,
                                      l.ctypes.data_as(C.POINTER(C.c_float)), f.ctypes.data_as(C.POINTER(C.c_float)),
                                      pdf.ctypes.data_as(C.POINTER(C.c_float)),
                                      ok.ctypes.data_as(C.POINTER(C.c_uint8)))
        return l, f, pdf, ok.astype(bool)


def texture_sample(pixels: np.ndarray, sampler, u: float, v: float, lod: float, srgb: bool):
    """(rgba, mip level count, last level's texel) of PreparedTexture::sample_lod."""
    a = _abi()
    px = np.ascontiguousarray(pixels)
    fmt = a.PT_PIXELS_RGBA8 if px.dtype == np.uint8 else a.PT_PIXELS_RGBA_F32
    if fmt == a.PT_PIXELS_RGBA_F32:
        px = np.ascontiguousarray(px, dtype=np.float32)
    t = a.pt_texture(px.shape[1], px.shape[0], fmt, px.ctypes.data, sampler.mag_filter, sampler.min_filter,
                     sampler.wrap_s, sampler.wrap_t)
    out = np.zeros(4, np.float32)
    top = np.zeros(4, np.float32)
    levels = C.c_uint32()
    lib().oracle_texture_sample(C.addressof(t), u, v, lod, 1 if srgb else 0, out.ctypes.data_as(C.POINTER(C.c_float)),
                                C.byref(levels), top.ctypes.data_as(C.POINTER(C.c_float)))
    return out, levels.value, top


def raycast(scene, opts):
    """RenderBackend::Raycast render of a PreparedScene (every shading
    mode): (HDR (h, w, 4) f32, RGBA8 (h, w, 4) u8)."""
    from oxideav_render_b200.scene import Camera
    w, h, aa = max(opts.width, 1), max(opts.height, 1), int(opts.aa)
    cam = Camera.resolve(scene, opts, w * aa, h * aa)
    desc = scene.to_desc(opts)
    c = cam.to_c()
    o = opts.to_raycast_c(cam.near, cam.far)
    hdr = np.zeros((h, w, 4), np.float32)
    rgba = np.zeros((h, w, 4), np.uint8)
    st = lib().oracle_raycast(C.addressof(desc.desc), C.addressof(c), C.addressof(o),
                              hdr.ctypes.data_as(C.POINTER(C.c_float)), rgba.ctypes.data_as(C.POINTER(C.c_uint8)))
    if st != 0:
        raise ValueError("options outside the raycast backend's range")
    return hdr, rgba


def gltf_brdf(base, metallic: float, roughness: float, f0_dielectric: float, n, v, l):
    """src/brdf.rs: (BrdfParams (c_diff, f0, alpha), eval(n, v, l))."""
    f3 = C.c_float * 3
    params, out = (C.c_float * 7)(), f3()
    lib().oracle_gltf_brdf(f3(*base), C.c_float(metallic), C.c_float(roughness), C.c_float(f0_dielectric),
                           f3(*n), f3(*v), f3(*l), params, out)
    return (tuple(params[0:3]), tuple(params[3:6]), params[6]), tuple(out)


def gltf_d_ggx(n_dot_h: float, alpha: float) -> float:
    lib().oracle_gltf_d_ggx.restype = C.c_float
    return lib().oracle_gltf_d_ggx(C.c_float(n_dot_h), C.c_float(alpha))


def gltf_schlick(f0, v_dot_h: float):
    f3 = C.c_float * 3
    out = f3()
    lib().oracle_gltf_schlick(f3(*f0), C.c_float(v_dot_h), out)
    return tuple(out)


def texture_mips(pixels: np.ndarray, srgb: bool) -> np.ndarray:
    """Every level of one mip chain (build_mips), concatenated, (n, 4) f32."""
    a = _abi()
    px = np.ascontiguousarray(pixels)
    fmt = a.PT_PIXELS_RGBA8 if px.dtype == np.uint8 else a.PT_PIXELS_RGBA_F32
    if fmt == a.PT_PIXELS_RGBA_F32:
        px = np.ascontiguousarray(px, dtype=np.float32)
    t = a.pt_texture(px.shape[1], px.shape[0], fmt, px.ctypes.data, 0, 0, 0, 0)
    n = lib().oracle_texture_mips(C.addressof(t), 1 if srgb else 0, None, 0)
    out = np.zeros((n, 4), np.float32)
    lib().oracle_texture_mips(C.addressof(t), 1 if srgb else 0, out.ctypes.data_as(C.POINTER(C.c_float)), n)
    return out


def sobol_owen_4d(index: int, seed: int) -> np.ndarray:
    out = np.zeros(4, np.float32)
    lib().oracle_sobol_owen_4d(index, seed, out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def sobol_owen_4d_many(n: int, seed: int) -> np.ndarray:
    out = np.zeros((n, 4), np.float32)
    for i in range(n):
        lib().oracle_sobol_owen_4d(i, seed, out[i].ctypes.data_as(C.POINTER(C.c_float)))
    return out
