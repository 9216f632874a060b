"""The C-ABI library loads on a machine without a GPU and exports exactly the
entry points include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

from fusion_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"FB_API\s+[\w\s\*]+?\b(fb_\w+)\s*\(", src))
    return names


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 30
    for n in sorted(names):
        assert hasattr(lib, n), n
    # the Python binding covers the whole C ABI
    assert names == set(_lib.exported_symbols())


def test_host_only_entry_points():
    lib = _lib.load()
    c = _lib.Config()
    lib.fb_default_config(ctypes.byref(c), 640, 480)
    assert (c.num_buckets, c.num_excess, c.num_blocks) == (1000000, 500000, 700000)
    assert abs(c.voxel_size - 0.006) < 1e-9 and list(c.iters) == [10, 5, 3]
    assert lib.fb_session_bytes(ctypes.byref(c)) > 700000 * 512 * 8
    assert lib.fb_status_string(_lib.FB_EINVAL) == b"invalid argument"
    h2d, d2h = ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.fb_frame_transfer_bytes(ctypes.byref(c), ctypes.byref(h2d), ctypes.byref(d2h)) == 0
    assert h2d.value == 640 * 480 * 5 and 0 < d2h.value < 1024
    bad = _lib.Config()
    assert lib.fb_session_bytes(ctypes.byref(bad)) == 0
    out = ctypes.c_void_p()
    assert lib.fb_session_create(ctypes.byref(bad), None, ctypes.byref(out)) == _lib.FB_EINVAL
