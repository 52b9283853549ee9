"""One small end-to-end render on cuda:0, checked against the oracle.

Renders the 36-triangle Cornell box at 32x32 / 8 spp through the C ABI and
requires (a) bit-exact camera-ray hits and (b) HDR parity (MAE <= 2e-3,
PSNR >= 45 dB) against the CPU restatement. Raises on any mismatch.
"""
from __future__ import annotations

import sys

import numpy as np


def run() -> None:
    from . import api, testscenes as ts
    from .options import PathTraceOptions
    from .scene import Camera

    oracle = sys.modules.get("pt_oracle")
    if oracle is None:
        import __graft_entry__
        oracle = __graft_entry__.load_oracle()
    scene, opts = ts.cornell_c0()
    opts = opts.replace(width=32, height=32, path_trace=PathTraceOptions(samples_per_pixel=8, max_bounces=8))
    ctx = api.Context(0)
    t = api.PathTracer(ctx)
    t.sync(scene, opts)
    t.refine(8)
    hdr = t.hdr()
    g_dev, tb = t.debug_primary_hits(0)

    desc = scene.to_desc(opts)
    osc = oracle.OracleScene(desc)
    ot = oracle.OracleTracer(osc, Camera.resolve(scene, opts, 32, 32), opts)
    ot.refine(8)
    ref = ot.hdr()
    g_ref, t_ref, _ = ot.primary_hits(0)
    if not np.array_equal(g_dev, g_ref) or not np.array_equal(tb[..., 0][g_ref != 0xFFFFFFFF],
                                                              t_ref[g_ref != 0xFFFFFFFF]):
        raise AssertionError("camera-ray hits differ from the oracle")
    mae, psnr = ts.hdr_mae(hdr, ref), ts.hdr_psnr(hdr, ref)
    if not (mae <= 2e-3 and psnr >= 45.0):
        raise AssertionError(f"HDR parity failed: MAE {mae:.3g}, PSNR {psnr:.1f} dB")
    ext, shadow = t.ray_counts()
    print(f"smoke ok: MAE {mae:.2e} PSNR {psnr:.1f} dB, {ext} extension + {shadow} shadow rays, "
          f"{t.last_kernel_ms():.3f} ms")
    t.close()
    ctx.close()
