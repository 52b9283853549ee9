"""oxideav-render B200 path tracer: RenderBackend::PathTraceCuda.

A drop-in for oxideav-render's CPU PathTrace backend. The compute lives in
`_lib/libpt_b200.so` (hand-written CUDA for sm_100a behind the C ABI of
include/pt_b200.h); this package holds the host-side mirror of the
reference's interface (`PathTracer`, `PathTraceRenderer`, `RenderOptions`,
`PreparedScene`, `Camera`, test scenes and metrics) over that ABI.
"""
from . import abi, options, scene, testscenes  # noqa: F401
from .options import (BackgroundColor, CameraSpec, LightSpec, LightStrategy, PathTraceOptions, Projection,  # noqa
                      RenderBackend, RenderOptions, ShadingMode, ToneMap, radiance_key)
from .scene import Camera, Material, MaterialExt, PreparedScene, Primitive, Sampler, Texture, TextureRef  # noqa

__all__ = [
    "abi", "options", "scene", "testscenes", "BackgroundColor", "CameraSpec", "LightSpec", "LightStrategy",
    "PathTraceOptions", "Projection", "RenderBackend", "RenderOptions", "ShadingMode", "ToneMap", "radiance_key",
    "Camera", "Material", "MaterialExt", "PreparedScene", "Primitive", "Sampler", "Texture", "TextureRef",
]


def __getattr__(name):
    # The native bindings load lazily so the package imports on hosts
    # without a GPU (or before the library is built).
    if name in ("api", "native", "serve"):
        import importlib
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)
