"""Host-side scene preparation through the C ABI, without a GPU:
pt_debug_prepare_scene validates a pt_scene_desc and builds the device
image (textures, BVH, tables) on the host."""
import ctypes as C

import numpy as np

from oxideav_render_b200 import abi, native, testscenes as ts


def prepare(desc):
    lib = native.load()
    sec = (C.c_double * 4)()
    nb = C.c_uint64()
    st = lib.pt_debug_prepare_scene(C.byref(desc), sec, C.byref(nb))
    msg = (lib.pt_last_error(None) or b"").decode()
    return st, list(sec), nb.value, msg


def test_scenes_prepare_on_the_host():
    for scene, opts in (ts.cornell_c0(), ts.sphere_grid_c1(64, 2)):
        d = scene.to_desc(opts)
        st, sec, nbytes, _ = prepare(d.desc)
        assert st == abi.PT_OK
        assert sec[0] >= sec[2] >= 0.0 and nbytes > 0
    # More triangles, more device bytes. The SceneDesc owns the buffers its
    # pt_scene_desc points into, so it stays bound across the call.
    small_desc = ts.random_soup(1000, seed=1).to_desc(ts.pt_opts(8, 1, 1))
    large_desc = ts.random_soup(20000, seed=1).to_desc(ts.pt_opts(8, 1, 1))
    small = prepare(small_desc.desc)[2]
    large = prepare(large_desc.desc)[2]
    assert large > small


def test_bad_descriptors_are_rejected_with_a_message():
    scene, opts = ts.cornell_c0()
    d = scene.to_desc(opts)
    bad = abi.pt_scene_desc.from_buffer_copy(d.desc)
    bad.material_count = 0
    st, _, _, msg = prepare(bad)
    assert st == abi.PT_ERR_INVALID_ARG and "material" in msg
    item = abi.pt_draw_item.from_buffer_copy(d.desc.items[0])
    item.material = 10_000
    items = (abi.pt_draw_item * 1)(item)
    bad = abi.pt_scene_desc.from_buffer_copy(d.desc)
    bad.item_count = 1
    bad.items = C.cast(items, C.POINTER(abi.pt_draw_item))
    st, _, _, msg = prepare(bad)
    assert st == abi.PT_ERR_INVALID_ARG and "material index" in msg
    item.material = 0
    item.positions = C.POINTER(C.c_float)()
    items = (abi.pt_draw_item * 1)(item)
    bad.items = C.cast(items, C.POINTER(abi.pt_draw_item))
    st, _, _, msg = prepare(bad)
    assert st == abi.PT_ERR_INVALID_ARG and "positions" in msg


def test_an_empty_scene_prepares():
    scene, opts = ts.cornell_c0()
    d = scene.to_desc(opts)
    empty = abi.pt_scene_desc.from_buffer_copy(d.desc)
    empty.item_count = 0
    st, _, nbytes, _ = prepare(empty)
    assert st == abi.PT_OK and nbytes > 0
    assert np.isfinite(nbytes)
