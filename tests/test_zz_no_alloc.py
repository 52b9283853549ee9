"""pt_refine_noalloc: the refine pass for callers that cannot allocate device
memory inside a call (a frame loop that forbids cudaMalloc / cudaFree, or a
host whose memory all comes from its own pool). The caller owns the
accumulator; the library's per-wave samples go to a fixed scratch array.

The output must equal what pt_tracer_refine accumulates, on two calls in a
row (the second continues the sample sequence). Both paths run the same
kernels in the same order, so the tolerance here is exact equality.
"""
import ctypes as C

import numpy as np
import pytest

from oxideav_render_b200 import abi, api, testscenes as ts
from oxideav_render_b200.options import PathTraceOptions

pytestmark = pytest.mark.gpu


def test_noalloc_refine_matches_tracer_refine_on_two_calls(ctx):
    import torch

    scene, opts = ts.cornell_c0()
    opts = opts.replace(width=64, height=48, path_trace=PathTraceOptions(samples_per_pixel=8, max_bounces=6))
    t = api.PathTracer(ctx)
    t.sync(scene, opts)
    t.refine(3)
    ref3 = t.accum()
    t.refine(5)
    ref8 = t.accum()

    # The caller's own device buffer (here from torch's allocator).
    acc = torch.zeros((48, 64, 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    cam, o = t.camera.to_c(), opts.to_c()
    lib = ctx.lib
    st = lib.pt_refine_noalloc(ctx.ptr, t.scene_id, C.byref(cam), C.byref(o), 0, 3, C.c_void_p(acc.data_ptr()))
    ctx.check(st)
    first = acc.cpu().numpy()
    np.testing.assert_allclose(first, ref3, rtol=0, atol=0)
    st = lib.pt_refine_noalloc(ctx.ptr, t.scene_id, C.byref(cam), C.byref(o), 3, 5, C.c_void_p(acc.data_ptr()))
    ctx.check(st)
    np.testing.assert_allclose(acc.cpu().numpy(), ref8, rtol=0, atol=0)
    t.close()


def test_noalloc_rejects_images_beyond_its_scratch(ctx):
    import torch

    scene, opts = ts.cornell_c0()
    t = api.PathTracer(ctx)
    t.sync(scene, opts)
    big = opts.replace(width=2048, height=1024)
    cam, o = t.camera.to_c(), big.to_c()
    acc = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = ctx.lib.pt_refine_noalloc(ctx.ptr, t.scene_id, C.byref(cam), C.byref(o), 0, 1, C.c_void_p(acc.data_ptr()))
    assert st == abi.PT_ERR_INVALID_ARG
    assert b"1048576" in ctx.lib.pt_last_error(ctx.ptr)
    t.close()


def test_noalloc_rejects_bad_accumulators_before_any_launch(ctx):
    # A misaligned, host, or too-small accumulator is refused on the host
    # with PT_ERR_INVALID_ARG; nothing is launched, so nothing can fault.
    import torch

    scene, opts = ts.cornell_c0()
    opts = opts.replace(width=32, height=16, path_trace=PathTraceOptions(samples_per_pixel=2, max_bounces=4))
    t = api.PathTracer(ctx)
    t.sync(scene, opts)
    cam, o = t.camera.to_c(), opts.to_c()
    lib = ctx.lib
    acc = torch.zeros((16 * 32 * 4 + 2,), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    def call(ptr):
        return lib.pt_refine_noalloc(ctx.ptr, t.scene_id, C.byref(cam), C.byref(o), 0, 1, C.c_void_p(ptr))

    assert call(acc.data_ptr() + 8) == abi.PT_ERR_INVALID_ARG
    assert b"aligned" in lib.pt_last_error(ctx.ptr)
    host = np.zeros(16 * 32 * 4, np.float64)
    assert call(host.ctypes.data) == abi.PT_ERR_INVALID_ARG
    assert b"device" in lib.pt_last_error(ctx.ptr)
    # A dedicated 32-byte allocation given a 1024x1024 image (32 MiB of
    # accumulator): the allocation-range check refuses it.
    from cuda.bindings import runtime as rt

    err, small = rt.cudaMalloc(32)
    assert err == rt.cudaError_t.cudaSuccess
    try:
        big = opts.replace(width=1024, height=1024).to_c()
        st = lib.pt_refine_noalloc(ctx.ptr, t.scene_id, C.byref(cam), C.byref(big), 0, 1, C.c_void_p(int(small)))
        assert st == abi.PT_ERR_INVALID_ARG
        assert b"pixels" in lib.pt_last_error(ctx.ptr)
    finally:
        rt.cudaFree(small)
    # The checks leave the context usable: a good call still matches.
    acc.zero_()
    torch.cuda.synchronize()
    ctx.check(call(acc.data_ptr()))
    t.refine(1)
    np.testing.assert_array_equal(acc[: 16 * 32 * 4].cpu().numpy().reshape(16, 32, 4), t.accum())
    t.close()
