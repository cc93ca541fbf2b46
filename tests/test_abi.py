"""The C-ABI library loads, exports every entry point include/*.h declares,
and rejects bad arguments without a GPU."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import reef3d_b200 as r3d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(r3d_[A-Za-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = r3d.load_library()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    # the Python layer binds exactly the declared C-ABI
    assert set(r3d.EXPORTS) == set(names)


def test_footprint_and_bad_descriptors():
    r3d.load_library()
    b = r3d.footprint(256, 256, 256, r3d.FP32)
    assert 7 * 256 ** 3 * 4 < b < 7 * 300 ** 3 * 4
    d = r3d.make_desc(8, 8, 8, r3d.uniform_nodes(8), r3d.uniform_nodes(8), r3d.uniform_nodes(8))
    d.nx = 0
    out = ctypes.c_size_t()
    assert r3d._lib.r3d_footprint(ctypes.byref(d), ctypes.byref(out)) == r3d.R3D_EINVAL
    assert b"sizes" in r3d._lib.r3d_last_error(None)
    bad = r3d.uniform_nodes(8)[::-1].copy()
    d2 = r3d.make_desc(8, 8, 8, bad, r3d.uniform_nodes(8), r3d.uniform_nodes(8))
    assert r3d._lib.r3d_footprint(ctypes.byref(d2), ctypes.byref(out)) == r3d.R3D_EINVAL
    with pytest.raises(ValueError):
        r3d.make_desc(8, 8, 8, r3d.uniform_nodes(7), r3d.uniform_nodes(8), r3d.uniform_nodes(8))
    # picard flags: 0..3 accepted; other forms and negative iterations refused
    for f46, f47, rc in ((2, 10, r3d.R3D_OK), (1, 0, r3d.R3D_OK), (3, 10, r3d.R3D_OK), (4, 10, r3d.R3D_EINVAL),
                         (2, -1, r3d.R3D_EINVAL)):
        d3 = r3d.make_desc(8, 8, 8, r3d.uniform_nodes(8), r3d.uniform_nodes(8), r3d.uniform_nodes(8),
                           f46=f46, f47=f47)
        assert r3d._lib.r3d_footprint(ctypes.byref(d3), ctypes.byref(out)) == rc


def test_null_handle_calls_fail_cleanly():
    lib = r3d.load_library()
    assert lib.r3d_ls_step(None, 0.1) == r3d.R3D_EINVAL
    assert lib.r3d_upload(None, 0, None, 0) == r3d.R3D_EINVAL
    assert lib.r3d_destroy(None) == r3d.R3D_OK
