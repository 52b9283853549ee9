"""The C ABI: ctypes mirrors match the header's layout, and the built library
loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from oxideav_render_b200 import abi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = []
    for h in sorted(os.listdir(INCLUDE)):
        if h.endswith(".h"):
            text = open(os.path.join(INCLUDE, h)).read()
            names += re.findall(r"^PT_API\s+[\w\s\*]+?\b(pt_\w+)\s*\(", text, flags=re.M)
    return names


def test_struct_layout_matches_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pt_b200.h"', '#include "pt_b200_serve.h"',
             '#include "pt_b200_debug.h"', "int main(void) {"]
    for cls in abi.ABI_STRUCTS:
        n = cls.__name__
        lines.append(f'printf("{n} %zu\\n", sizeof({n}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{n}.{fname} %zu\\n", offsetof({n}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-I", INCLUDE, src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for cls in abi.ABI_STRUCTS:
        n = cls.__name__
        assert int(got[n]) == C.sizeof(cls), n
        for fname, _ in cls._fields_:
            assert int(got[f"{n}.{fname}"]) == getattr(cls, fname).offset, f"{n}.{fname}"


def test_library_exports_every_declared_symbol():
    lib = native.load()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
        assert n in native.SIGNATURES, f"{n} has no ctypes signature"
    assert lib.pt_abi_version() == 2


def test_create_without_a_device_fails_cleanly():
    """On a host without a GPU pt_create returns an error status (no crash)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    lib = native.load()
    p = C.c_void_p()
    st = lib.pt_create(C.byref(p), 0)
    assert st in (abi.PT_ERR_DEVICE, abi.PT_ERR_INVALID_ARG)
    assert lib.pt_last_error(None)
