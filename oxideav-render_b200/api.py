"""The reference's path-tracer interface over the CUDA library.

* `PathTracer` mirrors oxideav_render::pathtrace::PathTracer
  (src/pathtrace.rs:2369-2735): `sync` / `refine` / `samples` /
  `is_converged` / `image` / `hdr` / `set_environment` /
  `invalidate_scene` / `reset`, with the same reset rule and the same
  sample-index continuation, the accumulator living on the GPU.
* `PathTraceCudaRenderer` mirrors `PathTraceRenderer` (:2745-2782):
  `render` / `render_hdr` re-prepare the scene and take `samples_per_pixel`
  samples.
* `make_renderer(RenderBackend.PathTraceCuda)` is the one new match arm of
  `make_renderer` (src/lib.rs:174-180).

Scenes are `PreparedScene`s (the reference's `PreparedScene::build` output);
the camera is `Camera.resolve` of the options, exactly as the reference's
`sync` does.
"""
from __future__ import annotations

import ctypes as C
import weakref
from typing import Optional

import numpy as np

from . import abi, native
from .native import RenderError, check
from .options import RenderBackend, RenderOptions, radiance_key
from .scene import Camera, PreparedScene, SceneDesc


class Context:
    """One CUDA device (pt_context)."""

    def __init__(self, device: int = 0):
        self.lib = native.load()
        p = C.c_void_p()
        st = self.lib.pt_create(C.byref(p), device)
        if st != abi.PT_OK:
            raise RenderError(st, (self.lib.pt_last_error(None) or b"").decode())
        self.ptr = p
        self.device = device
        self._tracers = weakref.WeakSet()  # destroyed before the context

    def close(self):
        if getattr(self, "ptr", None):
            for t in list(self._tracers):
                t.close()
            self.lib.pt_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st: int):
        check(st, self.ptr)

    def upload(self, desc: SceneDesc) -> int:
        sid = C.c_uint32()
        self.check(self.lib.pt_scene_upload(self.ptr, C.byref(desc.desc), C.byref(sid)))
        return sid.value

    def release(self, scene_id: int) -> None:
        self.check(self.lib.pt_scene_release(self.ptr, scene_id))

    def refit(self, scene_id: int, desc: SceneDesc) -> None:
        """pt_scene_refit: resident scene `scene_id` becomes `desc` (same draw
        items and triangle counts), its BVH refitted on the device."""
        self.check(self.lib.pt_scene_refit(self.ptr, scene_id, C.byref(desc.desc)))

    def scene_bytes(self, scene_id: int) -> int:
        b = C.c_uint64()
        self.check(self.lib.pt_scene_device_bytes(self.ptr, scene_id, C.byref(b)))
        return b.value

    def bvh_stats(self, scene_id: int) -> dict:
        n, l, d = C.c_uint32(), C.c_uint32(), C.c_uint32()
        sah, sec = C.c_double(), C.c_double()
        self.check(self.lib.pt_scene_bvh_stats(self.ptr, scene_id, C.byref(n), C.byref(l), C.byref(d),
                                               C.byref(sah), C.byref(sec)))
        return {"nodes": n.value, "leaves": l.value, "max_depth": d.value, "sah_cost": sah.value,
                "build_seconds": sec.value}

    def set_bvh_builder(self, builder: int) -> None:
        """pt_set_bvh_builder: abi.PT_BVH_BUILD_AUTO / _HOST / _DEVICE / _DEVICE_PLOC."""
        self.check(self.lib.pt_set_bvh_builder(self.ptr, builder))

    def upload_seconds(self, scene_id: int) -> dict:
        """pt_scene_upload_seconds: where the scene's upload time went."""
        s = (C.c_double * 4)()
        self.check(self.lib.pt_scene_upload_seconds(self.ptr, scene_id, s))
        return {"host_image": s[0], "device_copy": s[1], "device_bvh": s[2], "total": s[3]}

    def scene_texels(self, scene_id: int) -> np.ndarray:
        """pt_debug_scene_texels: the scene's device texel pool, (n, 4) f32."""
        total = C.c_uint64()
        self.check(self.lib.pt_debug_scene_texels(self.ptr, scene_id, None, 0, C.byref(total)))
        out = np.zeros((total.value, 4), np.float32)
        self.check(self.lib.pt_debug_scene_texels(self.ptr, scene_id, out.ctypes.data_as(C.POINTER(C.c_float)),
                                                  total.value, C.byref(total)))
        return out

    def bvh_on_device(self, scene_id: int) -> bool:
        v = C.c_int()
        self.check(self.lib.pt_scene_bvh_on_device(self.ptr, scene_id, C.byref(v)))
        return bool(v.value)

    def set_schedule(self, schedule: int) -> None:
        self.check(self.lib.pt_set_schedule(self.ptr, schedule))

    def set_wave_slots(self, slots: int) -> None:
        self.check(self.lib.pt_set_wave_slots(self.ptr, slots))

    @staticmethod
    def _tune_dict(c: abi.pt_tune_choice) -> dict:
        return {name: getattr(c, name) for name, _ in abi.pt_tune_choice._fields_}

    def autotune(self, tracer: "PathTracer", samples: int = 0) -> dict:
        """pt_autotune: the fastest configuration for the tracer's scene class
        (measured on a scratch accumulator); later refines of that class use it."""
        c = abi.pt_tune_choice()
        self.check(self.lib.pt_autotune(self.ptr, tracer.ptr, int(samples), C.byref(c)))
        return self._tune_dict(c)

    def tune_lookup(self, tracer: "PathTracer") -> Optional[dict]:
        c = abi.pt_tune_choice()
        st = self.lib.pt_tune_lookup(self.ptr, tracer.ptr, C.byref(c))
        if st == abi.PT_ERR_NOT_FOUND:
            return None
        self.check(st)
        return self._tune_dict(c)

    def tune_reset(self) -> None:
        self.check(self.lib.pt_tune_reset(self.ptr))

    def set_wave_graphs(self, on: bool) -> None:
        self.check(self.lib.pt_set_wave_graphs(self.ptr, 1 if on else 0))

    def set_material_sort(self, on: bool) -> None:
        self.check(self.lib.pt_set_material_sort(self.ptr, 1 if on else 0))

    def set_wave_overlap(self, on) -> None:
        """Overlapped waves: False / 0 one wave at a time, True / 1 the default
        (three path-state arenas on three streams, or the scene class's tuned
        count), 2 or 3 that many arenas."""
        self.check(self.lib.pt_set_wave_overlap(self.ptr, int(on)))

    def set_shade_blocks(self, blocks_per_sm: int) -> None:
        """Occupancy of the wavefront shade kernel (3 or 4 blocks per SM)."""
        self.check(self.lib.pt_set_shade_blocks(self.ptr, int(blocks_per_sm)))

    def set_traversal(self, threads: int = 256, claim_chunk: int = 1) -> None:
        """pt_set_traversal: traversal kernels' block size (128 / 256) and
        queue entries per lane refill (1 / 2 / 4)."""
        self.check(self.lib.pt_set_traversal(self.ptr, int(threads), int(claim_chunk)))

    def set_node_width(self, extension: int, shadow: int) -> None:
        """BVH node layout (2 or 4 children) of extension and shadow rays."""
        self.check(self.lib.pt_set_node_width(self.ptr, extension, shadow))

    def fail_allocations(self, count: int) -> None:
        """pt_debug_fail_allocations: the next `count` device allocations of
        the context fail with PT_ERR_OOM (host-side injection, no CUDA call)."""
        self.check(self.lib.pt_debug_fail_allocations(self.ptr, int(count)))

    def set_stage_timing(self, on: bool) -> None:
        self.check(self.lib.pt_set_stage_timing(self.ptr, 1 if on else 0))

    def debug_sobol(self, n: int, seed: int) -> np.ndarray:
        out = np.zeros((n, 4), np.float32)
        self.check(self.lib.pt_debug_sobol(self.ptr, n, seed & 0xFFFFFFFF, out.ctypes.data_as(native.fp)))
        return out

    def debug_bsdf(self, ms: np.ndarray, v, ng, front: bool, dirs: np.ndarray, us: np.ndarray) -> np.ndarray:
        params = np.zeros(43, np.float32)
        params[:36] = ms
        params[36:39] = v
        params[39:42] = ng
        params[42] = 1.0 if front else 0.0
        dirs = np.ascontiguousarray(dirs, np.float32)
        us = np.ascontiguousarray(us, np.float32)
        n = dirs.shape[0]
        out = np.zeros((n, 12), np.float32)
        self.check(self.lib.pt_debug_bsdf(self.ptr, params.ctypes.data_as(native.fp), dirs.ctypes.data_as(native.fp),
                                          us.ctypes.data_as(native.fp), n, out.ctypes.data_as(native.fp)))
        return out


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class EnvironmentMap:
    """Equirectangular HDR environment (src/pathtrace.rs:1557-1741):
    scene-linear RGBA f32 pixels (h, w, 4), row 0 = +Y, times `intensity`."""

    def __init__(self, pixels: np.ndarray, intensity: float = 1.0):
        self.pixels = np.ascontiguousarray(pixels, dtype=np.float32)
        self.intensity = float(intensity)

    def to_c(self) -> abi.pt_environment:
        return abi.pt_environment(self.pixels.shape[1], self.pixels.shape[0],
                                  self.pixels.ctypes.data_as(C.POINTER(C.c_float)), self.intensity)


class PathTracer:
    """Progressive path tracer with a device-resident accumulator."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.lib = self.ctx.lib
        p = C.c_void_p()
        self.ctx.check(self.lib.pt_tracer_create(self.ctx.ptr, C.byref(p)))
        self.ptr = p
        self.ctx._tracers.add(self)
        self.opts = RenderOptions()
        self._scene = None
        self._scene_key = None
        self._scene_id = None
        self._desc = None
        self._dirty = True
        self._env = None
        self.camera: Optional[Camera] = None

    def close(self):
        if getattr(self, "ptr", None):
            if self.ctx.ptr:  # a tracer never outlives its context's native object
                self.lib.pt_tracer_destroy(self.ptr)
            self.ptr = None
        if self._scene_id is not None and self.ctx.ptr:
            self.ctx.release(self._scene_id)
            self._scene_id = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _prep_key(o: RenderOptions):
        # PrepareOptions::from_render_options (src/prepare.rs:137-146).
        return (o.time, o.animation, o.material_variant, o.use_scene_lights, o.light)

    def sync(self, scene: PreparedScene, opts: RenderOptions, refit: bool = False) -> bool:
        """PathTracer::sync: re-uploads the scene when invalidated or when a
        preparation input changed; resets exactly when radiance inputs change.
        With `refit` (animated frames), a scene with the same draw items and
        triangle counts as the uploaded one replaces it in place and its BVH
        is refitted instead of rebuilt (same images, cheaper per frame)."""
        key = (id(scene), self._prep_key(opts))
        need_prepare = self._dirty or self._scene is not scene or self._scene_key != key
        if need_prepare and refit and self._scene_id is not None:
            desc = scene.to_desc(opts)
            st = self.lib.pt_scene_refit(self.ctx.ptr, self._scene_id, C.byref(desc.desc))
            if st == abi.PT_OK:
                self._desc, self._scene, self._scene_key = desc, scene, key
                self._dirty = False
                self.lib.pt_tracer_invalidate_scene(self.ptr)
                need_prepare = False
            elif st != abi.PT_ERR_INVALID_ARG:
                self.ctx.check(st)
        if need_prepare:
            desc = scene.to_desc(opts)
            # The old scene goes first: its device memory and any background
            # host BVH build of it are freed before the new upload runs.
            if self._scene_id is not None:
                self.ctx.release(self._scene_id)
                self._scene_id = None
            sid = self.ctx.upload(desc)
            self._scene_id, self._desc, self._scene, self._scene_key = sid, desc, scene, key
            self._dirty = False
            self.lib.pt_tracer_invalidate_scene(self.ptr)
        w, h = max(opts.width, 1), max(opts.height, 1)
        self.camera = Camera.resolve(scene, opts, w, h)
        cam = self.camera.to_c()
        o = opts.to_c()
        reset = C.c_int()
        self.ctx.check(self.lib.pt_tracer_sync(self.ptr, self._scene_id, C.byref(cam), C.byref(o), C.byref(reset)))
        self.opts = opts
        return bool(reset.value)

    def sync_resident(self, scene_id: int, scene: PreparedScene, opts: RenderOptions) -> bool:
        """PathTracer::sync against a scene already uploaded to this context
        (Context.upload), which several tracers may share; the tracer does
        not own it (the caller releases it after the tracers are done).
        Resets exactly when the scene or a radiance input changed."""
        w, h = max(opts.width, 1), max(opts.height, 1)
        self.camera = Camera.resolve(scene, opts, w, h)
        cam = self.camera.to_c()
        o = opts.to_c()
        reset = C.c_int()
        self.ctx.check(self.lib.pt_tracer_sync(self.ptr, int(scene_id), C.byref(cam), C.byref(o), C.byref(reset)))
        self.opts = opts
        self._scene = None
        return bool(reset.value)

    def refine(self, samples: int) -> None:
        self.ctx.check(self.lib.pt_tracer_refine(self.ptr, int(samples)))

    def samples(self) -> int:
        s = C.c_uint32()
        self.ctx.check(self.lib.pt_tracer_samples(self.ptr, C.byref(s)))
        return s.value

    def is_converged(self) -> bool:
        c = C.c_int()
        self.ctx.check(self.lib.pt_tracer_is_converged(self.ptr, C.byref(c)))
        return bool(c.value)

    def reset(self) -> None:
        self.ctx.check(self.lib.pt_tracer_reset(self.ptr))

    def invalidate_scene(self) -> None:
        self._dirty = True
        self.ctx.check(self.lib.pt_tracer_invalidate_scene(self.ptr))

    def set_environment(self, env: Optional[EnvironmentMap]) -> None:
        self._env = env
        if env is None:
            self.ctx.check(self.lib.pt_tracer_set_environment(self.ptr, None))
        else:
            e = env.to_c()
            self.ctx.check(self.lib.pt_tracer_set_environment(self.ptr, C.byref(e)))

    def _dims(self):
        return max(self.opts.width, 1), max(self.opts.height, 1)

    def hdr(self) -> np.ndarray:
        w, h = self._dims()
        out = np.zeros((h, w, 4), np.float32)
        self.ctx.check(self.lib.pt_tracer_read_hdr(self.ptr, out.ctypes.data_as(native.fp), out.size))
        return out

    def image(self) -> np.ndarray:
        w, h = self._dims()
        out = np.zeros((h, w, 4), np.uint8)
        self.ctx.check(self.lib.pt_tracer_read_image(self.ptr, out.ctypes.data_as(native.u8p), out.size))
        return out

    def accum(self) -> np.ndarray:
        w, h = self._dims()
        out = np.zeros((h, w, 4), np.float64)
        self.ctx.check(self.lib.pt_tracer_read_accum(self.ptr, out.ctypes.data_as(native.dp), out.size))
        return out

    def ray_counts(self):
        e, s = C.c_uint64(), C.c_uint64()
        self.ctx.check(self.lib.pt_tracer_ray_counts(self.ptr, C.byref(e), C.byref(s)))
        return e.value, s.value

    def traversal_counts(self):
        n, t = C.c_uint64(), C.c_uint64()
        self.ctx.check(self.lib.pt_tracer_traversal_counts(self.ptr, C.byref(n), C.byref(t)))
        return n.value, t.value

    STAGES = ("raygen", "extend", "shade", "shadow", "accumulate", "megakernel", "sort", "nee")

    def stage_ms(self) -> dict:
        """Device ms per stage of the last refine (with stage timing on)."""
        out = np.zeros(len(self.STAGES), np.float32)
        self.ctx.check(self.lib.pt_tracer_stage_ms(self.ptr, out.ctypes.data_as(native.fp), len(self.STAGES)))
        return dict(zip(self.STAGES, (float(v) for v in out)))

    def traversal_split(self) -> dict:
        out = np.zeros(4, np.uint64)
        self.ctx.check(self.lib.pt_tracer_traversal_split(self.ptr, out.ctypes.data_as(native.u64p)))
        return {"ext_nodes": int(out[0]), "ext_tris": int(out[1]), "sh_nodes": int(out[2]), "sh_tris": int(out[3])}

    def last_kernel_ms(self) -> float:
        m = C.c_float()
        self.ctx.check(self.lib.pt_tracer_last_kernel_ms(self.ptr, C.byref(m)))
        return m.value

    @property
    def scene_id(self):
        return self._scene_id

    def debug_pattern(self, index: int, pattern: int) -> np.ndarray:
        w, h = self._dims()
        out = np.zeros((h, w, 4), np.float32)
        self.ctx.check(self.lib.pt_debug_pattern(self.ptr, index, pattern, out.ctypes.data_as(native.fp)))
        return out

    def debug_primary_hits(self, index: int = 0):
        w, h = self._dims()
        g = np.zeros((h, w), np.uint32)
        tb = np.zeros((h, w, 4), np.float32)
        self.ctx.check(self.lib.pt_debug_primary_hits(self.ptr, index, g.ctypes.data_as(native.u32p),
                                                      tb.ctypes.data_as(native.fp)))
        return g, tb


def refine_many(ctx: Context, tracers, samples) -> None:
    """Batched refine: tracers[i] gains samples[i] samples, all in shared
    waves (bit-identical to refining each alone)."""
    n = len(tracers)
    arr = (C.c_void_p * max(n, 1))(*[t.ptr for t in tracers])
    sp = (C.c_uint32 * max(n, 1))(*[int(s) for s in samples])
    ctx.check(ctx.lib.pt_tracer_refine_many(ctx.ptr, arr, sp, n))


def batch_counters(ctx: Context) -> dict:
    """pt_batch_counters + pt_batch_stage_ms: the last refine / batch as a whole."""
    v = np.zeros(9, np.uint64)
    ctx.check(ctx.lib.pt_batch_counters(ctx.ptr, v.ctypes.data_as(native.u64p)))
    st = np.zeros(len(PathTracer.STAGES), np.float32)
    ctx.check(ctx.lib.pt_batch_stage_ms(ctx.ptr, st.ctypes.data_as(native.fp), len(PathTracer.STAGES)))
    names = ("ext_rays", "shadow_rays", "ext_nodes", "ext_tris", "sh_nodes", "sh_tris", "samples", "waves",
             "rounds")
    out = {k: int(x) for k, x in zip(names, v)}
    out["stage_ms"] = dict(zip(PathTracer.STAGES, (float(x) for x in st)))
    return out


def batch_stats(ctx: Context) -> dict:
    ms, waves, rays = C.c_float(), C.c_uint32(), C.c_uint64()
    ctx.check(ctx.lib.pt_batch_stats(ctx.ptr, C.byref(ms), C.byref(waves), C.byref(rays)))
    return {"ms": ms.value, "waves": waves.value, "rays": rays.value}


class PathTraceCudaRenderer:
    """Renderer for RenderBackend::PathTraceCuda (PathTraceRenderer semantics)."""

    def __init__(self, ctx: Optional[Context] = None):
        self.tracer = PathTracer(ctx)

    def tracer_mut(self) -> PathTracer:
        return self.tracer

    def _run(self, scene: PreparedScene, opts: RenderOptions) -> None:
        self.tracer.invalidate_scene()
        self.tracer.sync(scene, opts)
        self.tracer.refine(max(opts.path_trace.samples_per_pixel, 1))

    def render(self, scene: PreparedScene, opts: RenderOptions) -> np.ndarray:
        self._run(scene, opts)
        return self.tracer.image()

    def render_hdr(self, scene: PreparedScene, opts: RenderOptions) -> np.ndarray:
        self._run(scene, opts)
        return self.tracer.hdr()

    def render_frame(self, scene: PreparedScene, opts: RenderOptions) -> np.ndarray:
        """`render` for consecutive frames of an animation: a frame with the
        same draw items and triangle counts as the previous one refits the
        resident scene's BVH instead of rebuilding it (the image is the one
        `render` gives)."""
        self.tracer.sync(scene, opts, refit=True)
        self.tracer.refine(max(opts.path_trace.samples_per_pixel, 1))
        return self.tracer.image()


class RaycastCudaRenderer:
    """Renderer for RenderBackend::Raycast (src/raycast.rs) on the device:
    every call prepares and uploads the scene (as the reference's
    `render` builds its PreparedScene and TraceScene per call), resolves the
    camera at the SSAA resolution, traces one ray per sample and resolves the
    frame. Every shading mode: the legacy ones (Flat, Gouraud, Phong with
    Whitted's shadow / mirror / refraction rays, Wireframe, NormalDebug,
    DepthDebug) and Pbr (glTF metallic-roughness at every hit with hard
    shadows, mirror reflection, refraction, see-through BLEND)."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.lib = self.ctx.lib

    def _run(self, scene: PreparedScene, opts: RenderOptions, hdr: bool) -> np.ndarray:
        opts.validate()
        w, h, aa = max(opts.width, 1), max(opts.height, 1), int(opts.aa)
        cam = Camera.resolve(scene, opts, w * aa, h * aa)
        desc = scene.to_desc(opts)
        sid = self.ctx.upload(desc)
        try:
            o = opts.to_raycast_c(cam.near, cam.far)
            c = cam.to_c()
            if hdr:
                out = np.zeros((h, w, 4), np.float32)
                st = self.lib.pt_raycast_render(self.ctx.ptr, sid, C.byref(c), C.byref(o),
                                                out.ctypes.data_as(C.POINTER(C.c_float)), out.size, None, 0)
            else:
                out = np.zeros((h, w, 4), np.uint8)
                st = self.lib.pt_raycast_render(self.ctx.ptr, sid, C.byref(c), C.byref(o), None, 0,
                                                out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size)
            self.ctx.check(st)
            return out
        finally:
            self.ctx.release(sid)

    def render(self, scene: PreparedScene, opts: RenderOptions) -> np.ndarray:
        return self._run(scene, opts, False)

    def render_hdr(self, scene: PreparedScene, opts: RenderOptions) -> np.ndarray:
        return self._run(scene, opts, True)


def make_renderer(backend: RenderBackend, ctx: Optional[Context] = None):
    """make_renderer (src/lib.rs:174-180) for the backends this library provides."""
    if backend == RenderBackend.PathTraceCuda:
        return PathTraceCudaRenderer(ctx)
    if backend == RenderBackend.Raycast:
        return RaycastCudaRenderer(ctx)
    raise NotImplementedError(f"{backend} is served by the reference crate, not by this library")


__all__ = ["Context", "EnvironmentMap", "PathTracer", "PathTraceCudaRenderer", "RaycastCudaRenderer", "make_renderer",
           "RenderError",
           "radiance_key"]
