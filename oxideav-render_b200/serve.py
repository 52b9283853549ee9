"""Render server over include/pt_b200_serve.h: continuous batching of
render requests over scenes kept resident in HBM.

A request is what `PathTraceRenderer::render_hdr` does for one (scene,
options) pair (src/pathtrace.rs:2745-2782), or `PathTracer::refine` + `hdr`
on a live accumulation (a continuation). The server's image for a request is
bit-identical to that of a `PathTracer` given the same scene, options and
sample count.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import abi, native
from .api import Context, EnvironmentMap, default_context
from .native import RenderError
from .options import RenderOptions
from .scene import Camera, PreparedScene


class RenderServer:
    def __init__(self, ctx: Optional[Context] = None, hbm_budget_bytes: int = 0, wave_slots: int = 0,
                 max_active: int = 0, megakernel: bool = False, pipeline_depth: int = 0, autotune: bool = False,
                 material_sort: bool = True, wave_overlap: bool = True, spatial_bvh: bool = True):
        self.ctx = ctx or default_context()
        self.lib = native.load()
        cfg = abi.pt_server_config(int(hbm_budget_bytes), int(wave_slots), int(max_active), 1 if megakernel else 0,
                                   int(pipeline_depth), 0, 0, 1 if autotune else 0, 0 if material_sort else 1,
                                   0 if wave_overlap else 1, 0 if spatial_bvh else 1)
        p = C.c_void_p()
        st = self.lib.pt_server_create(self.ctx.ptr, C.byref(cfg), C.byref(p))
        if st != abi.PT_OK:
            raise RenderError(st, (self.lib.pt_server_last_error(None) or b"").decode())
        self.ptr = p
        self._scenes = {}
        self._tickets = {}

    def _check(self, st: int):
        if st != abi.PT_OK:
            raise RenderError(st, (self.lib.pt_server_last_error(self.ptr) or b"").decode())

    def close(self):
        if getattr(self, "ptr", None):
            self.lib.pt_server_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def register(self, scene: PreparedScene, opts: RenderOptions, env: Optional[EnvironmentMap] = None) -> int:
        """Prepares `scene` under `opts`' preparation inputs (PrepareOptions::
        from_render_options, src/prepare.rs:137-146) and keeps its image."""
        desc = scene.to_desc(opts)
        key = C.c_uint32()
        e = env.to_c() if env is not None else None
        self._check(self.lib.pt_server_scene_register(self.ptr, C.byref(desc.desc), C.byref(e) if e else None,
                                                      C.byref(key)))
        self._scenes[key.value] = scene
        return key.value

    def unregister(self, key: int) -> None:
        self._check(self.lib.pt_server_scene_unregister(self.ptr, key))
        self._scenes.pop(key, None)

    def scene_info(self, key: int) -> dict:
        b, r = C.c_uint64(), C.c_int()
        self._check(self.lib.pt_server_scene_info(self.ptr, key, C.byref(b), C.byref(r)))
        return {"device_bytes": b.value, "resident": bool(r.value)}

    def submit(self, key: int, opts: RenderOptions, samples: Optional[int] = None, deadline_ms: int = 0) -> int:
        """A new accumulation of `samples` (default: opts' samples_per_pixel).
        With `deadline_ms` > 0 the request fails with PT_ERR_TIMEOUT when it
        has not finished that many ms after this call."""
        scene = self._scenes[key]
        w, h = max(opts.width, 1), max(opts.height, 1)
        cam = Camera.resolve(scene, opts, w, h)
        n = opts.path_trace.samples_per_pixel if samples is None else samples
        req = abi.pt_server_request(key, int(n), 0, cam.to_c(), opts.to_c(), int(deadline_ms))
        t = C.c_uint64()
        self._check(self.lib.pt_server_submit(self.ptr, C.byref(req), C.byref(t)))
        self._tickets[t.value] = (h, w)
        return t.value

    def submit_continuation(self, ticket: int, samples: int, deadline_ms: int = 0) -> int:
        """`samples` more on the accumulator of `ticket` (PathTracer::refine)."""
        req = abi.pt_server_request()
        req.samples = int(samples)
        req.continues = int(ticket)
        req.deadline_ms = int(deadline_ms)
        t = C.c_uint64()
        self._check(self.lib.pt_server_submit(self.ptr, C.byref(req), C.byref(t)))
        self._tickets[t.value] = self._tickets[ticket]
        return t.value

    @staticmethod
    def _stats(st: abi.pt_request_stats) -> dict:
        return {"queue_ms": st.queue_ms, "latency_ms": st.latency_ms, "width": st.width, "height": st.height,
                "samples": st.samples, "waves": st.waves}

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(hdr (h, w, 4) float32, stats dict) once the request finished;
        None when it is still running when `timeout_ms` (>= 0) runs out.
        Raises RenderError with the request's own failure (cancelled, its
        deadline passed, out of memory, ...)."""
        h, w = self._tickets[ticket]
        out = np.empty((h, w, 4), np.float32)
        st = abi.pt_request_stats()
        rc = self.lib.pt_server_wait(self.ptr, ticket, int(timeout_ms), out.ctypes.data_as(native.fp), out.size,
                                     C.byref(st))
        if rc == abi.PT_ERR_NOT_READY or (rc == abi.PT_ERR_TIMEOUT and timeout_ms >= 0 and self.poll_status(ticket)
                                          == abi.PT_ERR_NOT_READY):
            return None
        self._check(rc)
        return out, self._stats(st)

    def poll_status(self, ticket: int) -> int:
        """pt_server_poll's status: PT_ERR_NOT_READY while queued or running."""
        return self.lib.pt_server_poll(self.ptr, ticket, None, 0, None)

    def poll(self, ticket: int):
        """wait() without blocking: None while the request is queued or running."""
        h, w = self._tickets[ticket]
        out = np.empty((h, w, 4), np.float32)
        st = abi.pt_request_stats()
        rc = self.lib.pt_server_poll(self.ptr, ticket, out.ctypes.data_as(native.fp), out.size, C.byref(st))
        if rc == abi.PT_ERR_NOT_READY:
            return None
        self._check(rc)
        return out, self._stats(st)

    def cancel(self, ticket: int) -> None:
        """pt_server_cancel: the request ends with PT_ERR_CANCELLED."""
        self._check(self.lib.pt_server_cancel(self.ptr, ticket))

    def fail_allocations(self, count: int) -> None:
        """pt_server_debug_fail_allocations: the next `count` device
        allocations of the server fail as out of memory (host-side injection)."""
        self._check(self.lib.pt_server_debug_fail_allocations(self.ptr, int(count)))

    def release(self, ticket: int) -> None:
        self._check(self.lib.pt_server_release(self.ptr, ticket))
        self._tickets.pop(ticket, None)

    def stats(self) -> dict:
        s = abi.pt_server_stats()
        self._check(self.lib.pt_server_stats_get(self.ptr, C.byref(s)))
        return {name: getattr(s, name) for name, _ in abi.pt_server_stats._fields_}


__all__ = ["RenderServer"]
